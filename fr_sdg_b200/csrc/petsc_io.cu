// petsc_io.cu -- a device vector as one record of PETSc's binary Vec format.
//
// The reference writes solutions through PETSc's solution monitor
// (`-ts_monitor_solution binary:<file>`, read by TSSetFromOptions at
// petsc_solver_impl.hpp:557), and its post-processing tools read the file back
// record by record (tools/plot.py:109-129, tools/check_iso_vortex.py:215-233): a
// big-endian 4-byte class id 1211214 and a 4-byte length (both 8 bytes when
// PETSc uses 64-bit indices), then the values as big-endian doubles in the DMDA
// natural order, which is the order of the library's vectors.  Packing the record
// on the GPU turns the byte swap into one HBM-bound pass, so a host writer only
// copies the finished bytes to the file.
#include "../../include/frsdg.h"
#include "frsdg_internal.hpp"

#include <cstdint>

namespace frsdg
{
int report(int code, const char* msg);
int report_cuda(cudaError_t e, const char* what);
} // namespace frsdg

using namespace frsdg;

namespace
{
constexpr uint32_t kVecClassId = 1211214;  // PETSc VEC_FILE_CLASSID

__device__ __forceinline__ uint64_t swap64(uint64_t v)
{
    const uint32_t lo = static_cast<uint32_t>(v), hi = static_cast<uint32_t>(v >> 32);
    return (static_cast<uint64_t>(__byte_perm(lo, 0, 0x0123)) << 32) | __byte_perm(hi, 0, 0x0123);
}

// body[i] = byte-reversed bits of x[i]; the header is written by thread 0 of block 0
__global__ void __launch_bounds__(256) petsc_pack_kernel(const uint64_t* __restrict__ x, int64_t n,
                                                          int hdr_words, unsigned char* __restrict__ out)
{
    const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    if (tid == 0)
    {
        if (hdr_words == 1)
        {
            const uint32_t h[2] = {__byte_perm(kVecClassId, 0, 0x0123), __byte_perm(static_cast<uint32_t>(n), 0, 0x0123)};
            reinterpret_cast<uint2*>(out)[0] = make_uint2(h[0], h[1]);
        }
        else
        {
            reinterpret_cast<uint64_t*>(out)[0] = swap64(kVecClassId);
            reinterpret_cast<uint64_t*>(out)[1] = swap64(static_cast<uint64_t>(n));
        }
    }
    uint64_t* body = reinterpret_cast<uint64_t*>(out) + hdr_words;
    // four independent loads in flight per thread
    int64_t i = tid;
    for (; i + 3 * stride < n; i += 4 * stride)
    {
        const uint64_t a = __ldg(x + i), b = __ldg(x + i + stride), c = __ldg(x + i + 2 * stride),
                       d = __ldg(x + i + 3 * stride);
        body[i] = swap64(a);
        body[i + stride] = swap64(b);
        body[i + 2 * stride] = swap64(c);
        body[i + 3 * stride] = swap64(d);
    }
    for (; i < n; i += stride) body[i] = swap64(__ldg(x + i));
}

int header_bytes(int32_t index_bytes)
{
    return index_bytes == 4 ? 8 : index_bytes == 8 ? 16 : -1;
}
} // namespace

extern "C" int frsdg_petsc_vec_record_bytes(int64_t n, int32_t index_bytes, int64_t* bytes)
{
    const int hb = header_bytes(index_bytes);
    if (hb < 0) return report(FRSDG_ERR_ARG, "petsc record: index_bytes must be 4 or 8");
    if (n < 0 || !bytes) return report(FRSDG_ERR_ARG, "petsc record: negative length or null output");
    if (index_bytes == 4 && n > INT32_MAX)
        return report(FRSDG_ERR_ARG, "petsc record: length above 2^31-1 needs index_bytes = 8");
    *bytes = hb + 8 * n;
    return FRSDG_OK;
}

extern "C" int frsdg_petsc_vec_pack(const double* x, int64_t n, int32_t index_bytes, void* out, void* stream)
{
    int64_t total = 0;
    const int rc = frsdg_petsc_vec_record_bytes(n, index_bytes, &total);
    if (rc != FRSDG_OK) return rc;
    if (!out || (n > 0 && !x)) return report(FRSDG_ERR_ARG, "petsc record: null pointer");
    if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(out)) % 8)
        return report(FRSDG_ERR_ARG, "petsc record: x and out must be 8-byte aligned");
    constexpr int kThreads = 256;
    const int64_t want = (n + kThreads - 1) / kThreads;
    const int blocks = static_cast<int>(want < 1 ? 1 : want > 148 * 8 ? 148 * 8 : want);
    petsc_pack_kernel<<<blocks, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const uint64_t*>(x), n, header_bytes(index_bytes) / 8, static_cast<unsigned char*>(out));
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return report_cuda(e, "petsc_pack_kernel");
    return FRSDG_OK;
}
