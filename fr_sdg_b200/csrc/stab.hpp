// stab.hpp -- launch interface of the post-step stabilisation and the change of
// variables kernels.
#pragma once
#include "frsdg_internal.hpp"

namespace frsdg
{

struct StabArgs
{
    int    dim, Nx, Ny, per_x, per_y;
    int    apply_filter, apply_weno;
    double gam[3];        // WENO linear weights ((1-g)/2, g, (1-g)/2)
    double one_over_norm; // shock-sensor normalisation (filter.hpp:646-652)
    double theta, threshold;
    double F[kMaxN * kMaxN];
    double D[kMaxN * kMaxN];
    double w[kMaxN];
    const double* src;
    double*       dst;
};

cudaError_t launch_stab(int n, const StabArgs& a, cudaStream_t s);

// Post-step of a batch group: every tile of `tiles` is (instance in group, bx, by, -);
// inst[i] holds instance i's arguments (src = its last stage, dst = its state).
struct StabBatchArgs
{
    const StabArgs*   inst;
    const int*        inst_clock;  // batch index of each instance (its clock)
    const BatchClock* clock;
    const int4*       tiles;
    int               ntiles;
};
cudaError_t launch_stab_batch(int n, const StabBatchArgs& b, cudaStream_t s);
// tile of the 2D post-step kernel (elements per CTA along x and y)
void stab_tile_dims(int n, int* tx, int* ty);
cudaError_t launch_prim_to_cons(int dim, int n, int64_t nelem, const double* in, double* out, cudaStream_t s);

} // namespace frsdg
