// jacobi.hpp -- launchers of the element block-Jacobi preconditioner (jacobi.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace frsdg
{
// Largest element block the preconditioner inverts (p <= 5 in 2D: 4 (p+1)^2 <= 144);
// the FP64 block sits in one CTA's shared memory.
constexpr int kMaxBlockDofs = 144;

size_t block_inverse_smem(int n);
// inv[e] = inverse of the column-major n x n block blocks[e], in FP32; blocks with
// a zero pivot are counted in *singular and their inverse is left unwritten.
cudaError_t launch_block_inverse(const double* blocks, float* inv, int n, int64_t n_blocks, unsigned long long* singular,
                                 cudaStream_t s);
// z[e] = inv[e] r[e] for every element block.
cudaError_t launch_block_apply(const float* inv, const double* r, double* z, int n, int64_t n_blocks, cudaStream_t s);
} // namespace frsdg
