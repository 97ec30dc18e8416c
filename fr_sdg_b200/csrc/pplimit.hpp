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
    int       enabled;      // cfg.pp_limit
    int       fused;        // batch: the last stage's epilogue is the post-step (slots 2, 3 skip it)
};

// Positivity limiter over a batch group (affine 2D instances of one order): warp per
// element of the group's concatenated elements; the slot picks the buffer.
struct PPBatchArgs
{
    const PPArgs*      inst;        // per instance in the group
    const BatchInst2D* binst;       // their buffers
    const int64_t*     elem_begin;  // first element of each instance, ninst + 1 entries
    int                ninst;
    int64_t            nelem;
    BatchClock*        clock;       // per batch instance; the limiter pass of the state gathers its
                                    // max |v| + c into clock[i].amax (adaptive time steps)
    int                slot;        // 0-2: stage output b[slot]; 3: the state U after the post-step
                                    // (instances whose PPArgs::fused is set are skipped)
    int                pad_;
};
cudaError_t launch_pp_batch(int n, const PPBatchArgs& b, cudaStream_t s);
// advance the clocks of a batch by one step; count the instances still active
cudaError_t launch_batch_clock(BatchClock* clock, int count, int* active_count, cudaStream_t s);

cudaError_t launch_pp_limit(const PPArgs& a, cudaStream_t s);
// nodes of U (nelem elements) whose density is not positive and finite, added to *bad
cudaError_t launch_check_density(int dim, int n, int64_t nelem, const double* U, unsigned long long* bad,
                                 cudaStream_t s);
// y = s_rcp(x) (op 0) or s_sqrt(x) (op 1), elementwise
cudaError_t launch_device_math(int op, const double* x, double* y, int64_t n, cudaStream_t s);
// tc.cu: the split-precision tensor-core line contraction on its own (validation)
cudaError_t launch_tc_lines(int n, const float* v, const double* D, float* out, int64_t L, int* err, cudaStream_t s);

} // namespace frsdg
