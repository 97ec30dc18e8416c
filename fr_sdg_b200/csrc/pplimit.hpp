// pplimit.hpp -- launch interface of the positivity-preserving limiter (pplimit.cu).
#pragma once
#include "frsdg_internal.hpp"

namespace frsdg
{

struct PPArgs
{
    int       dim, n, gas_law;
    GasParams gas;
    double    eps0;         // cfg.pp_eps
    int64_t   nelem;        // elements of the vector
    int       Nx, Ny;       // 2D mesh (Ny: global rows) and
    int       row_base;     // global row of the vector's first element row
    double    w[kMaxN];     // GLL weights
    const double* detJ;     // 2D curved meshes: detJ per node [global elem][l n + k]; null: constant
    double*   U;            // state, limited in place
    float*    U32;          // optional FP32 copy of U, refreshed where U changes (2D)
};

cudaError_t launch_pp_limit(const PPArgs& a, cudaStream_t s);

} // namespace frsdg
