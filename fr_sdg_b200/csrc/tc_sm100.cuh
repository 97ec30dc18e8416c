// tc_sm100.cuh -- fifth-generation tensor cores (tcgen05) for the split-precision
// line contractions of the FP32 residual.
//
// A "line" is the N values of one flux component along one reference direction of
// one element (an element row or column).  Its derivative at the N nodes of the line
// is D v, D the N x N differentiation matrix.  A tile of L lines is one GEMM
//     out[L x 16] = A[L x 8] . B[8 x 16],   A[line][m] = v_m,  B[m][k] = D[k][m],
// with K padded from the line length to 8 and N to 16 by zeros (M = 128 takes N in
// steps of 16).  Each operand is split
// into a TF32 high part and a TF32 low part (x = hi + lo, hi = tf32(x),
// lo = tf32(x - hi)), and the product is accumulated in FP32 by three MMAs,
//     A_lo B_hi + A_hi B_lo + A_hi B_hi,
// the smallest terms first.  Every product of two TF32 values is exact in FP32, and
// hi + lo carries 22 significant bits, so the result has FP32 accuracy (the dropped
// A_lo B_lo term is 2^-22 of the product).
//
// Operands sit in shared memory in the canonical K-major layout without swizzle:
// core matrices of 8 rows x 16 bytes (4 TF32 values) stored as 128 contiguous bytes;
// the two 16-byte K chunks of a row group 128 bytes apart (leading byte offset),
// successive 8-row groups 256 bytes apart (stride byte offset).  One MMA of shape
// M = 128, N = 16, K = 8 per 128 lines and split term; the accumulator lives in TMEM
// (lane = line, column = derivative node) and is read back with tcgen05.ld by the
// warp that owns the lane quarter.
//
// Every wait here is bounded: the MMA-completion barrier is polled a fixed number of
// times, after which the caller sees `false` and flags the failure instead of spinning.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace frsdg
{
namespace tc
{

constexpr int kRowBytes   = 32;                  // 8 TF32 values per line
constexpr int kGroupBytes = 8 * kRowBytes;       // one 8-line group: two core matrices
constexpr int kTileLines  = 128;                 // lines per MMA (M)
constexpr int kTileBytes  = kTileLines * kRowBytes;
constexpr int kCols       = 16;                  // accumulator columns per MMA (N)
constexpr int kBBytes     = 2 * kGroupBytes;     // the B operand: 16 rows

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of value k (0..7) of line r in the canonical layout.
__host__ __device__ constexpr int line_offset(int r, int k)
{
    return (r >> 3) * kGroupBytes + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4;
}

__device__ __forceinline__ float to_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Shared-memory matrix descriptor: K-major, no swizzle, LBO 128 B, SBO 256 B.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr)
{
    uint64_t d = 0;
    d |= uint64_t((addr >> 4) & 0x3FFFu);
    d |= uint64_t(128u >> 4) << 16;
    d |= uint64_t(uint32_t(kGroupBytes) >> 4) << 32;
    d |= uint64_t(1) << 46;  // descriptor version of sm_100
    return d;                // base offset 0, legacy LBO mode, layout SWIZZLE_NONE (0)
}

// Instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B, both
// K-major, M = 128, N = 16, dense.
__host__ __device__ constexpr uint32_t idesc_tf32_m128_n16()
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);
}

// Split one line into its high and low TF32 parts at line r of the operand pair.
// v holds n <= 8 values; the rest of the 8 columns are written as zeros.
template <int N>
__device__ __forceinline__ void pack_line(unsigned char* hi, unsigned char* lo, int r, const float (&v)[N])
{
    static_assert(N <= 8, "lines of at most 8 nodes");
    float h[8], l[8];
#pragma unroll
    for (int k = 0; k < 8; ++k)
    {
        const float x = k < N ? v[k] : 0.0f;
        h[k] = to_tf32(x);
        l[k] = to_tf32(x - h[k]);
    }
#pragma unroll
    for (int c = 0; c < 2; ++c)
    {
        const int o = line_offset(r, 4 * c);
        *reinterpret_cast<float4*>(hi + o) = make_float4(h[4 * c], h[4 * c + 1], h[4 * c + 2], h[4 * c + 3]);
        *reinterpret_cast<float4*>(lo + o) = make_float4(l[4 * c], l[4 * c + 1], l[4 * c + 2], l[4 * c + 3]);
    }
}

// The B operand from an FP64 matrix: B[m][k] = D[k][m] as the K-major N x K operand,
// i.e. row k of the operand holds row k of D (rows N..15 zero).  16 threads (k = 0..15),
// one row each.
template <int N>
__device__ __forceinline__ void pack_matrix_row(unsigned char* hi, unsigned char* lo, int k, const double* D)
{
    float h[8], l[8];
#pragma unroll
    for (int m = 0; m < 8; ++m)
    {
        const double x = (k < N && m < N) ? D[k * N + m] : 0.0;
        const float xf = static_cast<float>(x);
        h[m] = to_tf32(xf);
        l[m] = to_tf32(static_cast<float>(x - static_cast<double>(h[m])));
    }
#pragma unroll
    for (int c = 0; c < 2; ++c)
    {
        const int o = line_offset(k, 4 * c);
        *reinterpret_cast<float4*>(hi + o) = make_float4(h[4 * c], h[4 * c + 1], h[4 * c + 2], h[4 * c + 3]);
        *reinterpret_cast<float4*>(lo + o) = make_float4(l[4 * c], l[4 * c + 1], l[4 * c + 2], l[4 * c + 3]);
    }
}

// Make this thread's generic-proxy shared-memory writes visible to the tensor core.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM allocation (one whole warp).  The column base is written to *dst (shared).
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Poll the barrier for the phase with parity `parity` (non-blocking test, a 64 ns sleep
// between polls); false after `limit` polls, i.e. after at least limit x 64 ns.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit)
{
    const uint32_t a = smem_u32(bar);
    for (int it = 0; it < limit; ++it)
    {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        __nanosleep(64);
    }
    return false;
}

// D[tmem] (+)= A . B, issued by one thread.
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, bool accumulate)
{
    const uint32_t idesc = idesc_tf32_m128_n16();
    const uint32_t acc = accumulate ? 1u : 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

// Arrive on `bar` once every MMA this thread issued so far has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// The split product of one 128-line tile: accumulator columns [col, col + 8) of the
// TMEM block `tmem` (16 columns written), operand tiles at the given shared addresses.
__device__ __forceinline__ void split_product(uint32_t tmem, uint32_t col, uint32_t a_hi, uint32_t a_lo, uint32_t b_hi,
                                              uint32_t b_lo)
{
    mma_tf32(tmem + col, smem_desc(a_lo), smem_desc(b_hi), false);
    mma_tf32(tmem + col, smem_desc(a_hi), smem_desc(b_lo), true);
    mma_tf32(tmem + col, smem_desc(a_hi), smem_desc(b_hi), true);
}

// Eight accumulator columns of this thread's TMEM lane (warp-collective; the warp
// reads lanes 32 (warp % 4) .. + 31).
__device__ __forceinline__ void load8(uint32_t tmem, uint32_t col, float (&o)[8])
{
    const uint32_t lane_base = (threadIdx.x / 32 % 4) * 32;
    const uint32_t addr = tmem + (lane_base << 16) + col;
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(addr)
                 : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) o[i] = __uint_as_float(r[i]);
}

} // namespace tc
} // namespace frsdg
