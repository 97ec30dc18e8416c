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
// (blocks spaced `stride` doubles apart: n * n for a block-diagonal array, 5 n * n for
// the diagonal slot of the five blocks of each element row)
cudaError_t launch_block_inverse(const double* blocks, int64_t stride, float* inv, int n, int64_t n_blocks,
                                 unsigned long long* singular, cudaStream_t s);
// off[e][s][.] = (float) blocks5[e][1 + s][.], s = 0..3
cudaError_t launch_offdiag_to_f32(const double* blocks5, float* off, int n, int64_t nel, cudaStream_t s);
// One symmetric red-black block Gauss-Seidel sweep z = M^-1 r on an Nx x Ny element grid
// (no periodic wrap): three launches, red / black / red.
cudaError_t launch_block_gs(const float* inv, const float* off, const double* r, double* z, int n, int Nx, int Ny,
                            cudaStream_t s);
// z[e] = inv[e] r[e] for every element block.
cudaError_t launch_block_apply(const float* inv, const double* r, double* z, int n, int64_t n_blocks, cudaStream_t s);
} // namespace frsdg
