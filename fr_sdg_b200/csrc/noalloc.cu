// noalloc.cu -- post-step stabilisation without any memory allocation.
//
// frsdg_post_step needs a copy of the solution while the WENO limiter runs (each
// element reads its neighbours' unlimited values), and the handle allocates that
// copy with cudaMalloc in frsdg_create.  Some callers cannot allocate device
// memory at the moment they want to limit a solution: code being recorded into a
// CUDA graph (cudaMalloc is not permitted during stream capture), code running
// under an external memory manager that forbids stray allocations, or a driver
// that may not synchronise the device.  frsdg_post_step_static serves them: it
// takes the configuration instead of a handle, builds the small operators on the
// host stack, and uses a fixed device array of this translation unit as the copy.
#include "../../include/frsdg.h"
#include "frsdg_internal.hpp"
#include "setup_ops.hpp"
#include "stab.hpp"

#include <cmath>
#include <mutex>
#include <vector>

namespace frsdg
{
int validate_config(const frsdg_config& c);
int report(int code, const char* msg);
int report_cuda(cudaError_t e, const char* what);
} // namespace frsdg

using namespace frsdg;

namespace
{
// Scratch copy of the solution for the WENO limiter, FRSDG_POST_STEP_STATIC_MAX_DOFS
// doubles (32 MiB).  It lives on every device that loads the library until the
// process exits.  Calls share it and it keeps the last call's contents; every call
// overwrites the part it reads before reading it, so nothing needs clearing.
static __device__ __align__(256) double g_post_step_scratch[FRSDG_POST_STEP_STATIC_MAX_DOFS];

// Device address of the scratch array in the calling thread's current CUDA context.
// The host-side name of a __device__ array is not a device address, and the address
// belongs to the context (a device reset makes a new one), so the lookups are cached
// per context, under a mutex: host threads may call concurrently.
using CtxGetCurrent = int (*)(void**);  // cuCtxGetCurrent, through the runtime's entry points

void* current_context()
{
    static CtxGetCurrent fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<CtxGetCurrent>(f);
    }();
    void* ctx = nullptr;
    if (!fn || fn(&ctx) != 0) return nullptr;
    return ctx;
}

struct ScratchEntry
{
    void*   ctx;
    double* ptr;
};
std::mutex g_scratch_mu;
std::vector<ScratchEntry> g_scratch;

int scratch_address(double** out)
{
    void* ctx = current_context();
    {
        std::lock_guard<std::mutex> lk(g_scratch_mu);
        for (const ScratchEntry& e : g_scratch)
            if (ctx && e.ctx == ctx)
            {
                *out = e.ptr;
                return FRSDG_OK;
            }
    }
    // first call in this context (or no context yet: the lookup creates the primary one)
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_post_step_scratch);
    if (e != cudaSuccess) return report_cuda(e, "cudaGetSymbolAddress(post-step scratch)");
    ctx = current_context();
    if (ctx)
    {
        std::lock_guard<std::mutex> lk(g_scratch_mu);
        bool seen = false;
        for (ScratchEntry& x : g_scratch)
            if (x.ctx == ctx)
            {
                x.ptr = static_cast<double*>(p);
                seen = true;
            }
        if (!seen) g_scratch.push_back({ctx, static_cast<double*>(p)});
    }
    *out = static_cast<double*>(p);
    return FRSDG_OK;
}
} // namespace

extern "C" int frsdg_post_step_static(const frsdg_config* cfg, double* U, void* stream)
{
    if (!cfg || !U) return report(FRSDG_ERR_ARG, "null argument");
    if (reinterpret_cast<uintptr_t>(U) & 15) return report(FRSDG_ERR_ARG, "device pointers must be 16-byte aligned");
    int rc = validate_config(*cfg);
    if (rc) return rc;
    if (cfg->pp_limit)
        return report(FRSDG_ERR_UNSUPPORTED, "frsdg_post_step_static: the positivity limiter needs a handle");
    const int n = cfg->poly_deg + 1;
    const int Nx = cfg->n_elems[0], Ny = cfg->dim == 2 ? cfg->n_elems[1] : 1;
    const int64_t ntot = int64_t(Nx) * Ny * (cfg->dim == 2 ? 4 * n * n : 3 * n);
    if (ntot > FRSDG_POST_STEP_STATIC_MAX_DOFS)
        return report(FRSDG_ERR_ARG, "frsdg_post_step_static: solution larger than FRSDG_POST_STEP_STATIC_MAX_DOFS");
    if (!cfg->apply_filter && !cfg->apply_weno) return FRSDG_OK;

    StabArgs s{};
    s.dim = cfg->dim;
    s.Nx = Nx;
    s.Ny = Ny;
    s.per_x = cfg->bc[FRSDG_LEFT].kind == FRSDG_BC_PERIODIC;
    s.per_y = cfg->dim == 2 && cfg->bc[FRSDG_TOP].kind == FRSDG_BC_PERIODIC;
    s.apply_filter = cfg->apply_filter;
    s.apply_weno = cfg->apply_weno;
    const double g = cfg->weno_gamma;
    s.gam[0] = (1 - g) * 0.5;
    s.gam[1] = g;
    s.gam[2] = (1 - g) * 0.5;
    const double dmin = std::fmin(s.gam[0], std::fmin(s.gam[1], s.gam[2]));
    s.one_over_norm = 1.0 / (std::pow(std::fabs(1.0 / dmin - 1.0), cfg->shock_theta) + 3.0 - 1.0);
    s.theta = cfg->shock_theta;
    s.threshold = cfg->shock_threshold;
    double x[kMaxN], dL[kMaxN], dR[kMaxN];
    ref_element_into(cfg->poly_deg, cfg->radau_corr, x, s.w, s.D, dL, dR);
    filter_matrix_into(cfg->poly_deg, x, s.w, cfg->filt_cut_off, cfg->filt_strength, cfg->filt_alpha, s.F);
    s.dst = U;
    s.src = U;

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cfg->apply_weno && !cfg->apply_filter)
    {
        // the limiter reads neighbours: limit from a copy into U
        double* scratch = nullptr;
        if ((rc = scratch_address(&scratch))) return rc;
        cudaError_t e = cudaMemcpyAsync(scratch, U, sizeof(double) * ntot, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return report_cuda(e, "post-step copy");
        s.src = scratch;
    }
    cudaError_t e = launch_stab(n, s, st);
    if (e != cudaSuccess) return report_cuda(e, "post-step launch");
    return FRSDG_OK;
}
