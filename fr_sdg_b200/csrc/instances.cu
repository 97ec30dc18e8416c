// instances.cu -- explicit instantiation of the residual kernels for one number of
// GLL points per direction, FRSDG_N (set by the build, 2..10), in FP64, in
// complex FP64 and (2D) in FP32.  Compiling one translation unit per N keeps the build parallel.
#include "residual1d.cuh"
#include "residual2d.cuh"

#ifndef FRSDG_N
#error "FRSDG_N must be defined"
#endif

namespace frsdg
{
template cudaError_t launch_fr2d<double, FRSDG_N>(int, int, int, const Fr2dArgs&, cudaStream_t);
template cudaError_t launch_fr2d<cplx, FRSDG_N>(int, int, int, const Fr2dArgs&, cudaStream_t);
template cudaError_t launch_fr2d<float, FRSDG_N>(int, int, int, const Fr2dArgs&, cudaStream_t);
template cudaError_t launch_fr1d<double, FRSDG_N>(int, int, const Fr1dArgs&, cudaStream_t);
template cudaError_t launch_fr1d<cplx, FRSDG_N>(int, int, const Fr1dArgs&, cudaStream_t);
template cudaError_t launch_fr2d_batch<double, FRSDG_N>(int, int, int, const Fr2dBatchArgs&, int, cudaStream_t, int*);
template cudaError_t launch_fr2d_batch<float, FRSDG_N>(int, int, int, const Fr2dBatchArgs&, int, cudaStream_t, int*);
} // namespace frsdg
