// capi.cu -- implementation of the C ABI in include/frsdg.h.
//
// The handle plays the role of the reference's PhysicsEvaluator + PetscSolver pair
// (physics_evaluator.hpp:158-318, petsc_solver_impl.hpp:444-755): it owns the
// reference element, the filter, the cached curved metrics, the boundary data
// and every workspace, and it turns each PETSc callback into one kernel launch.
#include "../../include/frsdg.h"
#include "device_math.cuh"
#include "frsdg_internal.hpp"
#include "setup_ops.hpp"
#include "jacobi.hpp"
#include "handle.hpp"
#include "pplimit.hpp"
#include "stab.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

using namespace frsdg;

namespace frsdg
{
// explicit instantiations live in residual2d_n*.cu / residual1d.cu
#define FRSDG_DECL(S, N)                                                                                       \
    extern template cudaError_t launch_fr2d<S, N>(int, int, int, const Fr2dArgs&, cudaStream_t);              \
    extern template cudaError_t launch_fr1d<S, N>(int, int, const Fr1dArgs&, cudaStream_t);
#define FRSDG_DECL_ALL(S)                                                                                      \
    FRSDG_DECL(S, 2) FRSDG_DECL(S, 3) FRSDG_DECL(S, 4) FRSDG_DECL(S, 5) FRSDG_DECL(S, 6) FRSDG_DECL(S, 7)    \
    FRSDG_DECL(S, 8) FRSDG_DECL(S, 9) FRSDG_DECL(S, 10)
FRSDG_DECL_ALL(double)
FRSDG_DECL_ALL(cplx)
#define FRSDG_DECL2(S, N) extern template cudaError_t launch_fr2d<S, N>(int, int, int, const Fr2dArgs&, cudaStream_t);
FRSDG_DECL2(float, 2) FRSDG_DECL2(float, 3) FRSDG_DECL2(float, 4) FRSDG_DECL2(float, 5) FRSDG_DECL2(float, 6)
FRSDG_DECL2(float, 7) FRSDG_DECL2(float, 8) FRSDG_DECL2(float, 9) FRSDG_DECL2(float, 10)
} // namespace frsdg

namespace
{
// Last error of the calling thread, in a fixed buffer so that reporting an error
// never allocates.
thread_local char g_err[256];

int fail(int code, const char* msg)
{
    std::snprintf(g_err, sizeof(g_err), "%s", msg);
    return code;
}
int cuda_fail(cudaError_t e, const char* what)
{
    std::snprintf(g_err, sizeof(g_err), "%s: %s", what, cudaGetErrorString(e));
    return FRSDG_ERR_CUDA;
}

template <class S> cudaError_t dispatch2d(int n, int gas, int riem, int geo, const Fr2dArgs& a, cudaStream_t s)
{
    switch (n)
    {
        case 2: return launch_fr2d<S, 2>(gas, riem, geo, a, s);
        case 3: return launch_fr2d<S, 3>(gas, riem, geo, a, s);
        case 4: return launch_fr2d<S, 4>(gas, riem, geo, a, s);
        case 5: return launch_fr2d<S, 5>(gas, riem, geo, a, s);
        case 6: return launch_fr2d<S, 6>(gas, riem, geo, a, s);
        case 7: return launch_fr2d<S, 7>(gas, riem, geo, a, s);
        case 8: return launch_fr2d<S, 8>(gas, riem, geo, a, s);
        case 9: return launch_fr2d<S, 9>(gas, riem, geo, a, s);
        case 10: return launch_fr2d<S, 10>(gas, riem, geo, a, s);
        default: return cudaErrorInvalidValue;
    }
}
template <class S> cudaError_t dispatch1d(int n, int gas, int riem, const Fr1dArgs& a, cudaStream_t s)
{
    switch (n)
    {
        case 2: return launch_fr1d<S, 2>(gas, riem, a, s);
        case 3: return launch_fr1d<S, 3>(gas, riem, a, s);
        case 4: return launch_fr1d<S, 4>(gas, riem, a, s);
        case 5: return launch_fr1d<S, 5>(gas, riem, a, s);
        case 6: return launch_fr1d<S, 6>(gas, riem, a, s);
        case 7: return launch_fr1d<S, 7>(gas, riem, a, s);
        case 8: return launch_fr1d<S, 8>(gas, riem, a, s);
        case 9: return launch_fr1d<S, 9>(gas, riem, a, s);
        case 10: return launch_fr1d<S, 10>(gas, riem, a, s);
        default: return cudaErrorInvalidValue;
    }
}

} // namespace

namespace frsdg
{
// Configuration checks shared by frsdg_create and the allocation-free entry point.
int validate_config(const frsdg_config& c)
{
    if (c.dim != 1 && c.dim != 2) return fail(FRSDG_ERR_ARG, "dim must be 1 or 2");
    if (c.poly_deg < 1 || c.poly_deg > 9) return fail(FRSDG_ERR_ARG, "poly_deg must be in [1, 9]");
    if (c.n_elems[0] < 2 || (c.dim == 2 && c.n_elems[1] < 2))
        return fail(FRSDG_ERR_ARG, "n_elems must be >= 2 in every direction");
    if (!(c.box_length[0] > 0.0) || (c.dim == 2 && !(c.box_length[1] > 0.0)))
        return fail(FRSDG_ERR_ARG, "box_length must be positive");
    if (c.gas_law != FRSDG_GAS_IDEAL && c.gas_law != FRSDG_GAS_VDW) return fail(FRSDG_ERR_ARG, "unknown gas_law");
    if (c.riemann != FRSDG_RUSANOV && c.riemann != FRSDG_HLLC) return fail(FRSDG_ERR_ARG, "unknown riemann scheme");
    if (!(c.gamma > 1.0)) return fail(FRSDG_ERR_ARG, "gamma must be > 1");
    if (c.dim == 2 && (c.geometry < 0 || c.geometry > FRSDG_GEOM_SINE_WARP)) return fail(FRSDG_ERR_ARG, "unknown geometry");
    if (c.coord_sys == FRSDG_COORD_RADIAL && c.dim != 1) return fail(FRSDG_ERR_UNSUPPORTED, "radial coordinates are 1D only");
    const int nb = c.dim == 2 ? 4 : 2;
    for (int d = 0; d < nb; ++d)
        if (c.bc[d].kind < 0 || c.bc[d].kind > FRSDG_BC_PRESSURE_OUTLET) return fail(FRSDG_ERR_ARG, "unknown bc kind");
    auto per = [&](int a, int b) { return c.bc[a].kind == FRSDG_BC_PERIODIC || c.bc[b].kind == FRSDG_BC_PERIODIC; };
    auto both = [&](int a, int b) { return c.bc[a].kind == FRSDG_BC_PERIODIC && c.bc[b].kind == FRSDG_BC_PERIODIC; };
    if (per(FRSDG_LEFT, FRSDG_RIGHT) && !both(FRSDG_LEFT, FRSDG_RIGHT))
        return fail(FRSDG_ERR_ARG, "periodic x needs both LEFT and RIGHT periodic");
    if (c.dim == 2 && per(FRSDG_TOP, FRSDG_BOTTOM) && !both(FRSDG_TOP, FRSDG_BOTTOM))
        return fail(FRSDG_ERR_ARG, "periodic y needs both TOP and BOTTOM periodic");
    if (c.dim == 1)
        for (int d = 0; d < 2; ++d)
            if (c.bc[d].kind > FRSDG_BC_DIRICHLET) return fail(FRSDG_ERR_UNSUPPORTED, "1D supports outflow, wall, periodic, dirichlet");
    if (c.apply_filter && c.filt_cut_off == c.poly_deg)
        return fail(FRSDG_ERR_ARG, "filter cut-off equal to poly_deg gives 0/0 in the filter strength");
    if (c.apply_weno && (c.weno_gamma > 1.0 || c.weno_gamma < 0.0)) return fail(FRSDG_ERR_ARG, "weno_gamma must be in [0,1]");
    if (!(c.csd_eps > 0.0)) return fail(FRSDG_ERR_ARG, "csd_eps must be positive");
    if (c.pp_limit && !(c.pp_eps > 0.0)) return fail(FRSDG_ERR_ARG, "pp_eps must be positive");
    return FRSDG_OK;
}

int report(int code, const char* msg) { return fail(code, msg); }
int report_cuda(cudaError_t e, const char* what) { return cuda_fail(e, what); }
} // namespace frsdg

// Element count and vector length of the vectors the entry points see.
static int64_t local_nelem(const frsdg_handle* h) { return h->win_rows ? int64_t(h->Nx) * h->win_rows : h->nelem; }
static int64_t local_ntot(const frsdg_handle* h) { return local_nelem(h) * h->ndofs; }
static void apply_window(const frsdg_handle* h, Fr2dArgs& a)
{
    if (!h->win_rows) return;
    a.Ny = h->win_rows;
    a.per_y = 0;  // periodic neighbours arrive as ghost rows
    a.row_base = h->win_base;
    a.row_begin = h->win_begin;
    a.row_end = h->win_end;
}

static void free_handle(frsdg_handle* h)
{
    if (!h) return;
    cudaFree(h->d_metrics);
    cudaFree(h->d_xnorm);
    cudaFree(h->d_ynorm);
    cudaFree(h->d_bxy);
    cudaFree(h->d_detJ);
    cudaFree(h->d_post);
    cudaFree(h->d_work);
    cudaFree(h->d_stage);
    cudaFree(h->d_bad);
    cudaFree(h->d_blocks);
    cudaFree(h->d_inv);
    cudaFree(h->d_singular);
    cudaFree(h->d_blocks5);
    cudaFree(h->d_off);
    for (cudaStream_t& q : h->hst)
        if (q) cudaStreamDestroy(q);
    for (cudaEvent_t& ev : h->hev)
        if (ev) cudaEventDestroy(ev);
    delete h;
}

template <class T> static int upload(T** dst, const std::vector<T>& v)
{
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(dst), sizeof(T) * (v.empty() ? 1 : v.size()));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
    if (!v.empty())
    {
        e = cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy");
    }
    return FRSDG_OK;
}

extern "C" {

int frsdg_abi_version(void) { return FRSDG_ABI_VERSION; }
const char* frsdg_last_error(void) { return g_err; }

int frsdg_config_default(frsdg_config* c)
{
    if (!c) return fail(FRSDG_ERR_ARG, "null config");
    std::memset(c, 0, sizeof(*c));
    c->dim = 2;
    c->poly_deg = 3;
    c->n_elems[0] = c->n_elems[1] = 10;
    c->box_length[0] = c->box_length[1] = 1.0;
    c->radau_corr = 0.0;
    c->gas_law = FRSDG_GAS_IDEAL;
    c->riemann = FRSDG_RUSANOV;
    c->gamma = 1.4;
    c->R_spec = 287.05;
    c->vdw_a = 161.94;
    c->vdw_b = 0.001265;
    c->coord_sys = FRSDG_COORD_CARTESIAN;
    c->geometry = FRSDG_GEOM_CARTESIAN;
    c->geom_profile = FRSDG_PROFILE_FLAT;
    for (int d = 0; d < 4; ++d) c->bc[d].kind = FRSDG_BC_OUTFLOW;
    c->apply_filter = 0;
    c->filt_cut_off = 2;
    c->filt_strength = 32;
    c->filt_alpha = 36.0;
    c->apply_weno = 0;
    c->weno_gamma = 0.998;
    c->shock_theta = 1.0;
    c->shock_threshold = 0.8;
    c->cond_sys = 0;
    c->csd_eps = 1e-7;
    c->pp_limit = 0;
    c->mixed_tc = 0;
    c->pp_eps = 1e-13;
    return FRSDG_OK;
}

int frsdg_reference_element(int32_t p, double c, double* nodes, double* w, double* D, double* dL, double* dR)
{
    try
    {
        const RefElem r = build_ref_element(p, c);
        if (nodes) std::memcpy(nodes, r.x.data(), sizeof(double) * r.n);
        if (w) std::memcpy(w, r.w.data(), sizeof(double) * r.n);
        if (D) std::memcpy(D, r.D.data(), sizeof(double) * r.n * r.n);
        if (dL) std::memcpy(dL, r.dL.data(), sizeof(double) * r.n);
        if (dR) std::memcpy(dR, r.dR.data(), sizeof(double) * r.n);
        return FRSDG_OK;
    }
    catch (const std::exception& e)
    {
        return fail(FRSDG_ERR_ARG, e.what());
    }
}

int frsdg_filter_matrix(int32_t p, int32_t cut_off, int32_t strength, double alpha, double* F)
{
    try
    {
        const RefElem r = build_ref_element(p, 0.0);
        const auto    f = build_filter_matrix(r, cut_off, strength, alpha);
        std::memcpy(F, f.data(), sizeof(double) * f.size());
        return FRSDG_OK;
    }
    catch (const std::exception& e)
    {
        return fail(FRSDG_ERR_ARG, e.what());
    }
}

int frsdg_create(const frsdg_config* cfg, frsdg_handle** out)
{
    if (!cfg || !out) return fail(FRSDG_ERR_ARG, "null argument");
    *out = nullptr;
    int rc = validate_config(*cfg);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    {
        cudaGetLastError();
        return fail(FRSDG_ERR_NODEVICE, "no CUDA device visible");
    }
    auto* h = new frsdg_handle();
    h->cfg = *cfg;
    cudaGetDevice(&h->device);
    try
    {
        h->re = build_ref_element(cfg->poly_deg, cfg->radau_corr);
    }
    catch (const std::exception& e)
    {
        delete h;
        return fail(FRSDG_ERR_ARG, e.what());
    }
    const int n = h->re.n;
    h->n = n;
    h->Nx = cfg->n_elems[0];
    h->Ny = cfg->dim == 2 ? cfg->n_elems[1] : 1;
    h->ndofs = cfg->dim == 2 ? 4 * n * n : 3 * n;
    h->nelem = int64_t(h->Nx) * h->Ny;
    h->ntot = h->nelem * h->ndofs;

    Ops ops{};
    for (int q = 0; q < n * n; ++q) ops.D[q] = h->re.D[q];
    for (int q = 0; q < n; ++q) { ops.dL[q] = h->re.dL[q]; ops.dR[q] = h->re.dR[q]; ops.csi[q] = h->re.x[q]; }
    for (int q = 0; q < n * n; ++q) ops.Df[q] = static_cast<float>(ops.D[q]);
    for (int q = 0; q < n; ++q) { ops.dLf[q] = static_cast<float>(ops.dL[q]); ops.dRf[q] = static_cast<float>(ops.dR[q]); }
    const GasParams gas{cfg->gamma, cfg->gas_law == FRSDG_GAS_VDW ? cfg->vdw_a : 0.0,
                        cfg->gas_law == FRSDG_GAS_VDW ? cfg->vdw_b : 0.0};
    const bool per_x = cfg->bc[FRSDG_LEFT].kind == FRSDG_BC_PERIODIC;
    const bool per_y = cfg->dim == 2 && cfg->bc[FRSDG_TOP].kind == FRSDG_BC_PERIODIC;

    rc = upload(&h->d_bad, std::vector<unsigned long long>(1, 0ull));
    if (rc != FRSDG_OK)
    {
        free_handle(h);
        return rc;
    }

    if (cfg->dim == 2)
    {
        const int Nx = h->Nx, Ny = h->Ny;
        GeometryMap geom(*cfg);
        const double hx = 1.0 / double(Nx), hy = 1.0 / double(Ny);
        auto comp_x = [&](int i, int k) { return hx * (double(i) + 0.5 * (1.0 + h->re.x[k])); };
        auto comp_y = [&](int j, int l) { return hy * (double(j) + 0.5 * (1.0 + h->re.x[l])); };
        // composite metrics of physics_evaluator.hpp:282-305
        auto metrics = [&](double cx, double cy, double m[4]) {
            const GeomJacobian g = geom.jacobian(cx, cy);
            const double dcsi_dr = 0.5 / double(Nx), deta_ds = 0.5 / double(Ny);
            const double dx_dr = g.dx_dcsi * dcsi_dr, dy_dr = g.dy_dcsi * dcsi_dr;
            const double dx_ds = g.dx_deta * deta_ds, dy_ds = g.dy_deta * deta_ds;
            const double detJ = dx_dr * dy_ds - dx_ds * dy_dr;
            m[0] = dy_ds / detJ;
            m[1] = -dx_ds / detJ;
            m[2] = -dy_dr / detJ;
            m[3] = dx_dr / detJ;
        };
        Fr2dArgs& a = h->a2;
        a.Nx = Nx;
        a.Ny = Ny;
        a.row_base = 0;
        a.row_begin = 0;
        a.row_end = Ny;
        a.per_x = per_x;
        a.per_y = per_y;
        a.gas = gas;
        a.Lx = cfg->box_length[0];
        a.Ly = cfg->box_length[1];
        a.ops = ops;
        a.bad = h->d_bad;
        a.nd = 4 * n * n;
        a.exact_bc = cfg->jvp_exact_bc;
        a.tc = cfg->mixed_tc ? 1 : 0;
        a.jac_cmode = ((per_x && (Nx & 1)) || (per_y && (Ny & 1))) ? 1 : 0;
        for (int d = 0; d < 4; ++d)
        {
            a.bc[d].kind = cfg->bc[d].kind;
            for (int q = 0; q < 4; ++q) a.bc[d].state[q] = cfg->bc[d].state[q];
            for (int q = 0; q < 6; ++q) a.bc[d].params[q] = cfg->bc[d].params[q];
        }
        h->geo = geom.affine() ? GEO_AFFINE : GEO_CURVED;
        {
            double m[4];
            metrics(0.5, 0.5, m);
            a.xi_x = m[0]; a.xi_y = m[1]; a.eta_x = m[2]; a.eta_y = m[3];
            a.scale_x = std::sqrt(m[0] * m[0] + m[1] * m[1]);
            a.scale_y = std::sqrt(m[2] * m[2] + m[3] * m[3]);
        }
        try
        {
            if (h->geo == GEO_CURVED)
            {
                std::vector<double> mt(size_t(h->nelem) * n * n * 4);
                for (int j = 0; j < Ny; ++j)
                    for (int i = 0; i < Nx; ++i)
                        for (int l = 0; l < n; ++l)
                            for (int k = 0; k < n; ++k)
                                metrics(comp_x(i, k), comp_y(j, l),
                                        &mt[(((size_t(j) * Nx + i) * n + l) * n + k) * 4]);
                std::vector<double> xn(size_t(Nx + 1) * Ny * n * 2), yn(size_t(Nx) * (Ny + 1) * n * 2);
                for (int j = 0; j < Ny; ++j)
                    for (int I = 0; I <= Nx; ++I)
                        for (int l = 0; l < n; ++l)
                        {
                            const auto nn = geom.x_face_normal(comp_x(I, 0), comp_y(j, l));
                            const size_t o = ((size_t(j) * (Nx + 1) + I) * n + l) * 2;
                            xn[o] = nn.first;
                            xn[o + 1] = nn.second;
                        }
                for (int J = 0; J <= Ny; ++J)
                    for (int i = 0; i < Nx; ++i)
                        for (int k = 0; k < n; ++k)
                        {
                            const auto nn = geom.y_face_normal(comp_x(i, k), comp_y(J, 0));
                            const size_t o = ((size_t(J) * Nx + i) * n + k) * 2;
                            yn[o] = nn.first;
                            yn[o + 1] = nn.second;
                        }
                if ((rc = upload(&h->d_metrics, mt)) || (rc = upload(&h->d_xnorm, xn)) || (rc = upload(&h->d_ynorm, yn)))
                {
                    free_handle(h);
                    return rc;
                }
                if (cfg->pp_limit)
                {
                    // detJ of the composite map at every node: the positivity limiter's
                    // quadrature weights (physics_evaluator.hpp:282-305)
                    std::vector<double> dj(size_t(h->nelem) * n * n);
                    for (int j = 0; j < Ny; ++j)
                        for (int i = 0; i < Nx; ++i)
                            for (int l = 0; l < n; ++l)
                                for (int k = 0; k < n; ++k)
                                {
                                    const GeomJacobian g = geom.jacobian(comp_x(i, k), comp_y(j, l));
                                    const double dcsi_dr = 0.5 / double(Nx), deta_ds = 0.5 / double(Ny);
                                    dj[((size_t(j) * Nx + i) * n + l) * n + k] =
                                        (g.dx_dcsi * dcsi_dr) * (g.dy_deta * deta_ds) -
                                        (g.dx_deta * deta_ds) * (g.dy_dcsi * dcsi_dr);
                                }
                    if ((rc = upload(&h->d_detJ, dj)))
                    {
                        free_handle(h);
                        return rc;
                    }
                }
            }
            // boundary face points: LEFT, RIGHT (Ny*n each), TOP, BOTTOM (Nx*n each)
            std::vector<double> bxy(size_t(2 * Ny * n + 2 * Nx * n) * 2);
            size_t off[4];
            off[FRSDG_LEFT] = 0;
            off[FRSDG_RIGHT] = size_t(Ny) * n * 2;
            off[FRSDG_TOP] = size_t(2 * Ny) * n * 2;
            off[FRSDG_BOTTOM] = off[FRSDG_TOP] + size_t(Nx) * n * 2;
            for (int j = 0; j < Ny; ++j)
                for (int l = 0; l < n; ++l)
                {
                    const auto pl = geom.physical(comp_x(0, 0), comp_y(j, l));
                    const auto pr = geom.physical(comp_x(Nx, 0), comp_y(j, l));
                    bxy[off[FRSDG_LEFT] + (j * n + l) * 2] = pl.first;
                    bxy[off[FRSDG_LEFT] + (j * n + l) * 2 + 1] = pl.second;
                    bxy[off[FRSDG_RIGHT] + (j * n + l) * 2] = pr.first;
                    bxy[off[FRSDG_RIGHT] + (j * n + l) * 2 + 1] = pr.second;
                }
            for (int i = 0; i < Nx; ++i)
                for (int k = 0; k < n; ++k)
                {
                    const auto pb = geom.physical(comp_x(i, k), comp_y(0, 0));
                    const auto pt = geom.physical(comp_x(i, k), comp_y(Ny, 0));
                    bxy[off[FRSDG_BOTTOM] + (i * n + k) * 2] = pb.first;
                    bxy[off[FRSDG_BOTTOM] + (i * n + k) * 2 + 1] = pb.second;
                    bxy[off[FRSDG_TOP] + (i * n + k) * 2] = pt.first;
                    bxy[off[FRSDG_TOP] + (i * n + k) * 2 + 1] = pt.second;
                }
            if ((rc = upload(&h->d_bxy, bxy)))
            {
                free_handle(h);
                return rc;
            }
            for (int d = 0; d < 4; ++d) a.bxy[d] = h->d_bxy + off[d];
        }
        catch (const std::exception& e)
        {
            free_handle(h);
            return fail(FRSDG_ERR_NOMEM, e.what());
        }
        a.metrics = h->d_metrics;
        a.xnorm = h->d_xnorm;
        a.ynorm = h->d_ynorm;
    }
    else
    {
        Fr1dArgs& a = h->a1;
        a.N = h->Nx;
        a.per = per_x;
        a.gas = gas;
        a.h_elem = cfg->box_length[0] / cfg->n_elems[0];
        a.inv_jac = 2.0 / a.h_elem;
        a.radial = cfg->coord_sys == FRSDG_COORD_RADIAL;
        for (int d = 0; d < 2; ++d)
        {
            a.bc[d].kind = cfg->bc[d].kind;
            for (int q = 0; q < 4; ++q) a.bc[d].state[q] = cfg->bc[d].state[q];
        }
        a.ops = ops;
        a.bad = h->d_bad;
    }

    // positivity limiter
    {
        PPArgs& p = h->pp;
        p.dim = cfg->dim;
        p.n = n;
        p.gas_law = cfg->gas_law;
        p.gas = gas;
        p.eps0 = cfg->pp_eps;
        p.Nx = h->Nx;
        p.Ny = h->Ny;
        p.row_base = 0;
        for (int q = 0; q < n; ++q) p.w[q] = h->re.w[q];
        p.detJ = h->d_detJ;
        p.enabled = cfg->pp_limit;
    }

    // post-step stabilisation
    {
        StabArgs& s = h->st;
        s.dim = cfg->dim;
        s.Nx = h->Nx;
        s.Ny = h->Ny;
        s.per_x = per_x;
        s.per_y = per_y;
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
        const auto F = build_filter_matrix(h->re, cfg->filt_cut_off, cfg->filt_strength, cfg->filt_alpha);
        for (int q = 0; q < n * n; ++q) { s.F[q] = F[q]; s.D[q] = h->re.D[q]; h->a2.ops.F[q] = F[q]; }
        for (int q = 0; q < n; ++q) s.w[q] = h->re.w[q];
        if (cfg->apply_weno && !cfg->apply_filter)
        {
            cudaError_t e = cudaMalloc(&h->d_work, sizeof(double) * h->ntot);
            if (e != cudaSuccess)
            {
                free_handle(h);
                return cuda_fail(e, "cudaMalloc(post-step workspace)");
            }
        }
    }

    // operands of the fused stage epilogue (frsdg_rk_stage_fused)
    if (cfg->dim == 2)
    {
        PostArgs pa{};
        for (int q = 0; q < n; ++q) pa.w[q] = h->re.w[q];
        pa.pp_eps = cfg->pp_eps;
        pa.detJ = h->d_detJ;
        pa.amax = nullptr;
        cudaError_t e = cudaMalloc(&h->d_post, sizeof(PostArgs));
        if (e == cudaSuccess) e = cudaMemcpy(h->d_post, &pa, sizeof(PostArgs), cudaMemcpyHostToDevice);
        if (e != cudaSuccess)
        {
            free_handle(h);
            return cuda_fail(e, "stage epilogue operands");
        }
    }
    *out = h;
    return FRSDG_OK;
}

int frsdg_destroy(frsdg_handle* h)
{
    free_handle(h);
    return FRSDG_OK;
}

int frsdg_n_dofs(const frsdg_handle* h, int64_t* n)
{
    if (!h || !n) return fail(FRSDG_ERR_ARG, "null argument");
    *n = h->ntot;
    return FRSDG_OK;
}

} // extern "C"

namespace
{
int run_residual(frsdg_handle* h, int mode, double t, const double* U, const double* W, double* out, void* stream,
                 const StageArgs* stage = nullptr)
{
    if (!h || !U || !out) return fail(FRSDG_ERR_ARG, "null argument");
    if ((reinterpret_cast<uintptr_t>(U) | reinterpret_cast<uintptr_t>(out)) & 15)
        return fail(FRSDG_ERR_ARG, "device pointers must be 16-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    h->last = s;
    const bool cvar = (mode == MODE_IFUNC || mode == MODE_JVP) && h->cfg.cond_sys;
    const double hh = h->cfg.csd_eps;
    cudaError_t e;
    if (h->cfg.dim == 2)
    {
        Fr2dArgs a = h->a2;
        a.t = t;
        a.mode = mode;
        a.cond_sys = cvar;
        a.U = U;
        a.W = W;
        a.out = out;
        a.h = hh;
        a.inv_h = 1.0 / hh;
        a.sigma = h->jvp_sigma;
        if (stage) a.st = *stage;
        apply_window(h, a);
        if (mode == MODE_JVP) e = dispatch2d<cplx>(h->n, h->cfg.gas_law, h->cfg.riemann, h->geo, a, s);
        else e = dispatch2d<double>(h->n, h->cfg.gas_law, h->cfg.riemann, h->geo, a, s);
    }
    else
    {
        Fr1dArgs a = h->a1;
        a.t = t;
        a.mode = mode;
        a.cond_sys = cvar;
        a.U = U;
        a.W = W;
        a.out = out;
        a.h = hh;
        a.inv_h = 1.0 / hh;
        a.sigma = h->jvp_sigma;
        if (stage) a.st = *stage;
        if (mode == MODE_JVP) e = dispatch1d<cplx>(h->n, h->cfg.gas_law, h->cfg.riemann, a, s);
        else e = dispatch1d<double>(h->n, h->cfg.gas_law, h->cfg.riemann, a, s);
    }
    if (e != cudaSuccess) return cuda_fail(e, "residual launch");
    return FRSDG_OK;
}
} // namespace

extern "C" {

int frsdg_residual(frsdg_handle* h, double t, const double* U, double* R, void* stream)
{
    return run_residual(h, MODE_RESIDUAL, t, U, nullptr, R, stream);
}

int frsdg_rhs(frsdg_handle* h, double t, const double* U, double* rhs, void* stream)
{
    return run_residual(h, MODE_RHS, t, U, nullptr, rhs, stream);
}

int frsdg_ifunction(frsdg_handle* h, double t, const double* U, const double* U_t, double* F, void* stream)
{
    if (!U_t) return fail(FRSDG_ERR_ARG, "null U_t");
    if (reinterpret_cast<uintptr_t>(U_t) & 15) return fail(FRSDG_ERR_ARG, "device pointers must be 16-byte aligned");
    return run_residual(h, MODE_IFUNC, t, U, U_t, F, stream);
}

int frsdg_rk_stage(frsdg_handle* h, double t, const double* Us, const double* A, double alpha, const double* B,
                   double beta, double gamma, double* out, double* acc, double delta, void* stream)
{
    if (!h || !Us || !out) return fail(FRSDG_ERR_ARG, "null argument");
    if (out == Us) return fail(FRSDG_ERR_ARG, "frsdg_rk_stage: out must not alias Us");
    if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B) | reinterpret_cast<uintptr_t>(acc)) & 15)
        return fail(FRSDG_ERR_ARG, "device pointers must be 16-byte aligned");
    StageArgs st{A, B, acc, alpha, beta, gamma, delta, nullptr};
    return run_residual(h, MODE_STAGE, t, Us, nullptr, out, stream, &st);
}

int frsdg_jvp_prepare(frsdg_handle* h, double t, double sigma, const double* U)
{
    if (!h || !U) return fail(FRSDG_ERR_ARG, "null argument");
    h->jvp_t = t;
    h->jvp_sigma = sigma;
    h->jvp_U = U;
    return FRSDG_OK;
}

int frsdg_jvp(frsdg_handle* h, const double* V, double* JV, void* stream)
{
    if (!h || !V) return fail(FRSDG_ERR_ARG, "null argument");
    if (!h->jvp_U) return fail(FRSDG_ERR_ARG, "frsdg_jvp called before frsdg_jvp_prepare");
    if (reinterpret_cast<uintptr_t>(V) & 15) return fail(FRSDG_ERR_ARG, "device pointers must be 16-byte aligned");
    return run_residual(h, MODE_JVP, h->jvp_t, h->jvp_U, V, JV, stream);
}

// Residual pass of the FP32 instantiation (2D): U32 is a float state, out is
// float (out_f32) or double (the stage forms).
// The FP32 instantiation of the 2D kernel; in_f64: U is an FP64 state whose node
// primitives are recovered in FP64 (the mixed form), else an FP32 state.
static int run_residual_f32(frsdg_handle* h, int mode, double t, const void* U, bool in_f64, void* out, bool out_f32,
                            const StageArgs* stage, void* stream)
{
    if (h->cfg.dim != 2) return fail(FRSDG_ERR_UNSUPPORTED, "FP32 residual: 2D configurations only");
    if ((reinterpret_cast<uintptr_t>(U) | reinterpret_cast<uintptr_t>(out)) & 15)
        return fail(FRSDG_ERR_ARG, "device pointers must be 16-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    h->last = s;
    Fr2dArgs a = h->a2;
    a.t = t;
    a.mode = mode;
    a.cond_sys = 0;
    a.in_f64 = in_f64 ? 1 : 0;
    a.U = static_cast<const double*>(U);
    a.W = nullptr;
    a.out = out;
    a.out_f32 = out_f32 ? 1 : 0;
    if (stage) a.st = *stage;
    apply_window(h, a);
    const cudaError_t e = dispatch2d<float>(h->n, h->cfg.gas_law, h->cfg.riemann, h->geo, a, s);
    if (e != cudaSuccess) return cuda_fail(e, "FP32 residual launch");
    return FRSDG_OK;
}

int frsdg_residual_f32(frsdg_handle* h, double t, const float* U32, float* R32, void* stream)
{
    if (!h || !U32 || !R32) return fail(FRSDG_ERR_ARG, "null argument");
    return run_residual_f32(h, MODE_RESIDUAL, t, U32, false, R32, true, nullptr, stream);
}

int frsdg_rk_stage_mixed(frsdg_handle* h, double t, const double* Us, const double* A, double alpha, const double* B,
                         double beta, double gamma, double* out, double* acc, double delta, void* stream)
{
    if (!h || !Us || !out) return fail(FRSDG_ERR_ARG, "null argument");
    StageArgs st{A, B, acc, alpha, beta, gamma, delta, nullptr};
    return run_residual_f32(h, MODE_STAGE, t, Us, true, out, false, &st, stream);
}

static int run_pp_limit(frsdg_handle* h, double* U, float* U32, cudaStream_t s);

int frsdg_rk_stage_fused(frsdg_handle* h, double t, const double* Us, const double* A, double alpha, const double* B,
                         double beta, double gamma, double* out, double* acc, double delta, int32_t flags, void* stream)
{
    if (!h || !Us || !out) return fail(FRSDG_ERR_ARG, "null argument");
    if (out == Us) return fail(FRSDG_ERR_ARG, "frsdg_rk_stage_fused: out must not alias Us");
    if (flags & ~(FRSDG_STAGE_MIXED | FRSDG_STAGE_LIMIT | FRSDG_STAGE_POST_STEP))
        return fail(FRSDG_ERR_ARG, "frsdg_rk_stage_fused: unknown flags");
    if ((reinterpret_cast<uintptr_t>(Us) | reinterpret_cast<uintptr_t>(out) | reinterpret_cast<uintptr_t>(A) |
         reinterpret_cast<uintptr_t>(B) | reinterpret_cast<uintptr_t>(acc)) & 15)
        return fail(FRSDG_ERR_ARG, "device pointers must be 16-byte aligned");
    const bool mixed = (flags & FRSDG_STAGE_MIXED) != 0;
    const bool step = (flags & FRSDG_STAGE_POST_STEP) != 0;
    const bool limit = (step || (flags & FRSDG_STAGE_LIMIT)) && h->cfg.pp_limit;
    if (mixed && (h->cfg.dim != 2 || h->cfg.cond_sys))
        return fail(FRSDG_ERR_UNSUPPORTED, "frsdg_rk_stage_fused: the mixed form needs a 2D configuration without "
                                           "change of variables");
    StageArgs st{A, B, acc, alpha, beta, gamma, delta, nullptr};
    // the post-step is element-local unless it is the WENO limiter alone (the filter
    // overrides WENO when both are set)
    const bool local_step = h->cfg.apply_filter || !h->cfg.apply_weno;
    // the limiter alone after a stage runs as its own pass (measured faster than the
    // epilogue on the 1024^2 p = 5 blast: 2.44 against 2.70 ms per stage)
    if (h->cfg.dim == 2 && step && local_step)
    {
        int post = limit ? POST_PP : 0;
        if (step && h->cfg.apply_filter) post |= POST_FILTER;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        h->last = s;
        Fr2dArgs a = h->a2;
        a.t = t;
        a.mode = MODE_STAGE;
        a.cond_sys = 0;
        a.U = Us;
        a.W = nullptr;
        a.out = out;
        a.out_f32 = 0;
        a.in_f64 = mixed ? 1 : 0;
        a.st = st;
        a.post = post;
        a.pa = h->d_post;
        apply_window(h, a);
        const cudaError_t e = mixed ? dispatch2d<float>(h->n, h->cfg.gas_law, h->cfg.riemann, h->geo, a, s)
                                    : dispatch2d<double>(h->n, h->cfg.gas_law, h->cfg.riemann, h->geo, a, s);
        if (e != cudaSuccess) return cuda_fail(e, "fused stage launch");
        return FRSDG_OK;
    }
    // 1D, the limiter alone, or a post-step that reads neighbours: the stage, then the
    // separate passes
    int rc = mixed ? run_residual_f32(h, MODE_STAGE, t, Us, true, out, false, &st, stream)
                   : run_residual(h, MODE_STAGE, t, Us, nullptr, out, stream, &st);
    if (rc) return rc;
    if (step) return frsdg_post_step(h, out, stream);
    if (limit) return run_pp_limit(h, out, nullptr, static_cast<cudaStream_t>(stream));
    return FRSDG_OK;
}

int frsdg_set_row_window(frsdg_handle* h, int row_base, int rows, int row_begin, int row_end)
{
    if (!h) return fail(FRSDG_ERR_ARG, "null argument");
    if (h->cfg.dim != 2) return fail(FRSDG_ERR_UNSUPPORTED, "frsdg_set_row_window: 2D configurations only");
    if (rows == 0)
    {
        h->win_rows = h->win_base = h->win_begin = h->win_end = 0;
        return FRSDG_OK;
    }
    const int Ny = h->Ny;
    if (rows < 0 || row_begin < 0 || row_end <= row_begin || row_end > rows || rows > Ny + 2)
        return fail(FRSDG_ERR_ARG, "frsdg_set_row_window: need 0 <= row_begin < row_end <= rows <= Ny + 2");
    const int g0 = row_base + row_begin, g1 = row_base + row_end;
    if (g0 < 0 || g1 > Ny) return fail(FRSDG_ERR_ARG, "frsdg_set_row_window: computed rows outside the mesh");
    const bool per_y = h->cfg.bc[FRSDG_TOP].kind == FRSDG_BC_PERIODIC;
    // a side without a ghost row must be the physical edge; a ghost row across the
    // physical edge exists only for periodic meshes
    if (row_begin == 0 && (g0 != 0 || per_y))
        return fail(FRSDG_ERR_ARG, "frsdg_set_row_window: the bottom side needs a ghost row");
    if (row_end == rows && (g1 != Ny || per_y))
        return fail(FRSDG_ERR_ARG, "frsdg_set_row_window: the top side needs a ghost row");
    if (row_begin > 0 && g0 == 0 && !per_y)
        return fail(FRSDG_ERR_ARG, "frsdg_set_row_window: ghost row below a non-periodic bottom edge");
    if (row_end < rows && g1 == Ny && !per_y)
        return fail(FRSDG_ERR_ARG, "frsdg_set_row_window: ghost row above a non-periodic top edge");
    h->win_rows = rows;
    h->win_base = row_base;
    h->win_begin = row_begin;
    h->win_end = row_end;
    return FRSDG_OK;
}

int frsdg_jac_blocks(frsdg_handle* h, double t, double sigma, const double* U, double* blocks, void* stream)
{
    if (!h || !U || !blocks) return fail(FRSDG_ERR_ARG, "null argument");
    if (h->cfg.dim != 2) return fail(FRSDG_ERR_UNSUPPORTED, "frsdg_jac_blocks: 2D configurations only");
    if ((reinterpret_cast<uintptr_t>(U) | reinterpret_cast<uintptr_t>(blocks)) & 15)
        return fail(FRSDG_ERR_ARG, "device pointers must be 16-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    h->last = s;
    Fr2dArgs a = h->a2;
    a.t = t;
    a.mode = MODE_JAC;
    a.cond_sys = h->cfg.cond_sys;
    a.U = U;
    a.W = nullptr;
    a.out = blocks;
    a.h = h->cfg.csd_eps;
    a.inv_h = 1.0 / h->cfg.csd_eps;
    a.sigma = sigma;
    apply_window(h, a);
    const cudaError_t e = dispatch2d<cplx>(h->n, h->cfg.gas_law, h->cfg.riemann, h->geo, a, s);
    if (e != cudaSuccess) return cuda_fail(e, "Jacobian-block launch");
    return FRSDG_OK;
}

int frsdg_pc_setup(frsdg_handle* h, double t, double sigma, const double* U, void* stream)
{
    if (!h || !U) return fail(FRSDG_ERR_ARG, "null argument");
    if (h->cfg.dim != 2) return fail(FRSDG_ERR_UNSUPPORTED, "frsdg_pc_setup: 2D configurations only");
    const int nd = h->ndofs;
    if (nd > kMaxBlockDofs) return fail(FRSDG_ERR_UNSUPPORTED, "frsdg_pc_setup: element blocks above 144 DOFs (p > 5)");
    cudaError_t e;
    if (!h->d_blocks)
    {
        const size_t nb = size_t(h->nelem) * nd * nd;
        if ((e = cudaMalloc(&h->d_blocks, sizeof(double) * nb)) != cudaSuccess) return cuda_fail(e, "cudaMalloc(blocks)");
        if ((e = cudaMalloc(&h->d_inv, sizeof(float) * nb)) != cudaSuccess) return cuda_fail(e, "cudaMalloc(inverse blocks)");
        if ((e = cudaMalloc(&h->d_singular, sizeof(unsigned long long))) != cudaSuccess)
            return cuda_fail(e, "cudaMalloc(pivot flag)");
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if ((e = cudaMemsetAsync(h->d_singular, 0, sizeof(unsigned long long), s)) != cudaSuccess)
        return cuda_fail(e, "cudaMemsetAsync");
    int rc = frsdg_jac_blocks(h, t, sigma, U, h->d_blocks, stream);
    if (rc) return rc;
    if ((e = launch_block_inverse(h->d_blocks, int64_t(nd) * nd, h->d_inv, nd, local_nelem(h), h->d_singular, s)) !=
        cudaSuccess)
        return cuda_fail(e, "block-inverse launch");
    unsigned long long nsing = 0;
    if ((e = cudaMemcpyAsync(&nsing, h->d_singular, sizeof(nsing), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return cuda_fail(e, "pivot flag read");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "pc setup sync");
    if (nsing) return fail(FRSDG_ERR_ARG, "frsdg_pc_setup: singular element block (zero pivot)");
    h->pc_kind = 1;
    return FRSDG_OK;
}

int frsdg_jac_blocks5(frsdg_handle* h, double t, double sigma, const double* U, double* blocks5, void* stream)
{
    if (!h || !U || !blocks5) return fail(FRSDG_ERR_ARG, "null argument");
    if (h->cfg.dim != 2) return fail(FRSDG_ERR_UNSUPPORTED, "frsdg_jac_blocks5: 2D configurations only");
    if (h->win_rows) return fail(FRSDG_ERR_UNSUPPORTED, "frsdg_jac_blocks5: whole-mesh handles only (no row window)");
    const bool per_x = h->cfg.bc[FRSDG_LEFT].kind == FRSDG_BC_PERIODIC;
    const bool per_y = h->cfg.bc[FRSDG_TOP].kind == FRSDG_BC_PERIODIC;
    if ((per_x && h->Nx % 5) || (per_y && h->Ny % 5))
        return fail(FRSDG_ERR_UNSUPPORTED, "frsdg_jac_blocks5: periodic directions need a multiple of 5 elements");
    if ((reinterpret_cast<uintptr_t>(U) | reinterpret_cast<uintptr_t>(blocks5)) & 15)
        return fail(FRSDG_ERR_ARG, "device pointers must be 16-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    h->last = s;
    Fr2dArgs a = h->a2;
    a.t = t;
    a.mode = MODE_JAC;
    a.jac_cmode = 2;
    a.cond_sys = h->cfg.cond_sys;
    a.U = U;
    a.W = nullptr;
    a.out = blocks5;
    a.h = h->cfg.csd_eps;
    a.inv_h = 1.0 / h->cfg.csd_eps;
    a.sigma = sigma;
    const cudaError_t e = dispatch2d<cplx>(h->n, h->cfg.gas_law, h->cfg.riemann, h->geo, a, s);
    if (e != cudaSuccess) return cuda_fail(e, "Jacobian-block launch");
    return FRSDG_OK;
}

int frsdg_pc_setup_gs(frsdg_handle* h, double t, double sigma, const double* U, void* stream)
{
    if (!h || !U) return fail(FRSDG_ERR_ARG, "null argument");
    if (h->cfg.dim != 2) return fail(FRSDG_ERR_UNSUPPORTED, "frsdg_pc_setup_gs: 2D configurations only");
    if (h->cfg.bc[FRSDG_LEFT].kind == FRSDG_BC_PERIODIC || h->cfg.bc[FRSDG_TOP].kind == FRSDG_BC_PERIODIC)
        return fail(FRSDG_ERR_UNSUPPORTED, "frsdg_pc_setup_gs: non-periodic meshes only");
    const int nd = h->ndofs;
    if (nd > kMaxBlockDofs) return fail(FRSDG_ERR_UNSUPPORTED, "frsdg_pc_setup_gs: element blocks above 144 DOFs (p > 5)");
    cudaError_t e;
    const size_t nb = size_t(h->nelem) * nd * nd;
    if (!h->d_blocks5)
    {
        if ((e = cudaMalloc(&h->d_blocks5, sizeof(double) * 5 * nb)) != cudaSuccess) return cuda_fail(e, "cudaMalloc(blocks)");
        if ((e = cudaMalloc(&h->d_off, sizeof(float) * 4 * nb)) != cudaSuccess) return cuda_fail(e, "cudaMalloc(blocks)");
    }
    if (!h->d_inv && (e = cudaMalloc(&h->d_inv, sizeof(float) * nb)) != cudaSuccess)
        return cuda_fail(e, "cudaMalloc(inverse blocks)");
    if (!h->d_singular && (e = cudaMalloc(&h->d_singular, sizeof(unsigned long long))) != cudaSuccess)
        return cuda_fail(e, "cudaMalloc(pivot flag)");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if ((e = cudaMemsetAsync(h->d_singular, 0, sizeof(unsigned long long), s)) != cudaSuccess)
        return cuda_fail(e, "cudaMemsetAsync");
    int rc = frsdg_jac_blocks5(h, t, sigma, U, h->d_blocks5, stream);
    if (rc) return rc;
    if ((e = launch_block_inverse(h->d_blocks5, 5 * int64_t(nd) * nd, h->d_inv, nd, h->nelem, h->d_singular, s)) !=
        cudaSuccess)
        return cuda_fail(e, "block-inverse launch");
    if ((e = launch_offdiag_to_f32(h->d_blocks5, h->d_off, nd, h->nelem, s)) != cudaSuccess)
        return cuda_fail(e, "off-diagonal packing launch");
    unsigned long long nsing = 0;
    if ((e = cudaMemcpyAsync(&nsing, h->d_singular, sizeof(nsing), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return cuda_fail(e, "pivot flag read");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "pc setup sync");
    if (nsing) return fail(FRSDG_ERR_ARG, "frsdg_pc_setup_gs: singular element block (zero pivot)");
    h->pc_kind = 2;
    return FRSDG_OK;
}

int frsdg_pc_apply(frsdg_handle* h, const double* r, double* z, void* stream)
{
    if (!h || !r || !z) return fail(FRSDG_ERR_ARG, "null argument");
    if (!h->pc_kind) return fail(FRSDG_ERR_ARG, "frsdg_pc_apply called before frsdg_pc_setup");
    if (r == z) return fail(FRSDG_ERR_ARG, "frsdg_pc_apply: z must not alias r");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    h->last = s;
    const cudaError_t e = h->pc_kind == 2 ? launch_block_gs(h->d_inv, h->d_off, r, z, h->ndofs, h->Nx, h->Ny, s)
                                          : launch_block_apply(h->d_inv, r, z, h->ndofs, local_nelem(h), s);
    if (e != cudaSuccess) return cuda_fail(e, "block-apply launch");
    return FRSDG_OK;
}

// The positivity limiter over the handle's vectors (whole mesh or row window).
static int run_pp_limit(frsdg_handle* h, double* U, float* U32, cudaStream_t s)
{
    if (!h->cfg.pp_limit) return FRSDG_OK;
    PPArgs p = h->pp;
    p.U = U;
    p.U32 = U32;
    p.nelem = local_nelem(h);
    p.row_base = h->win_rows ? h->win_base : 0;
    const cudaError_t e = launch_pp_limit(p, s);
    if (e != cudaSuccess) return cuda_fail(e, "positivity-limiter launch");
    return FRSDG_OK;
}

int frsdg_pp_limit(frsdg_handle* h, double* U, float* U32, void* stream)
{
    if (!h || !U) return fail(FRSDG_ERR_ARG, "null argument");
    if ((reinterpret_cast<uintptr_t>(U) | reinterpret_cast<uintptr_t>(U32)) & 15)
        return fail(FRSDG_ERR_ARG, "device pointers must be 16-byte aligned");
    if (U32 && h->cfg.dim != 2) return fail(FRSDG_ERR_ARG, "frsdg_pp_limit: the FP32 copy is 2D only");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    h->last = s;
    return run_pp_limit(h, U, U32, s);
}

int frsdg_post_step(frsdg_handle* h, double* U, void* stream)
{
    if (!h || !U) return fail(FRSDG_ERR_ARG, "null argument");
    if (reinterpret_cast<uintptr_t>(U) & 15) return fail(FRSDG_ERR_ARG, "device pointers must be 16-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!h->cfg.apply_filter && !h->cfg.apply_weno)
    {
        h->last = s;
        return run_pp_limit(h, U, nullptr, s);
    }
    h->last = s;
    StabArgs a = h->st;
    a.dst = U;
    a.src = U;
    if (h->win_rows)
    {
        a.Ny = h->win_rows;
        a.per_y = 0;
    }
    if (h->d_work)
    {
        cudaError_t e = cudaMemcpyAsync(h->d_work, U, sizeof(double) * local_ntot(h), cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return cuda_fail(e, "post-step copy");
        a.src = h->d_work;
    }
    cudaError_t e = launch_stab(h->n, a, s);
    if (e != cudaSuccess) return cuda_fail(e, "post-step launch");
    return run_pp_limit(h, U, nullptr, s);
}

int frsdg_post_step_to(frsdg_handle* h, const double* src, double* dst, void* stream)
{
    if (!h || !src || !dst) return fail(FRSDG_ERR_ARG, "null argument");
    if ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15)
        return fail(FRSDG_ERR_ARG, "device pointers must be 16-byte aligned");
    if (src == dst) return fail(FRSDG_ERR_ARG, "frsdg_post_step_to: src and dst must not alias");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    h->last = s;
    if (!h->cfg.apply_filter && !h->cfg.apply_weno)
    {
        cudaError_t e = cudaMemcpyAsync(dst, src, sizeof(double) * local_ntot(h), cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return cuda_fail(e, "post-step copy");
        return run_pp_limit(h, dst, nullptr, s);
    }
    StabArgs a = h->st;
    a.src = src;
    a.dst = dst;
    if (h->win_rows)
    {
        a.Ny = h->win_rows;
        a.per_y = 0;
    }
    cudaError_t e = launch_stab(h->n, a, s);
    if (e != cudaSuccess) return cuda_fail(e, "post-step launch");
    return run_pp_limit(h, dst, nullptr, s);
}

int frsdg_prim_to_cons(frsdg_handle* h, const double* prim, double* cons, void* stream)
{
    if (!h || !prim || !cons) return fail(FRSDG_ERR_ARG, "null argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    h->last = s;
    cudaError_t e = launch_prim_to_cons(h->cfg.dim, h->n, local_nelem(h), prim, cons, s);
    if (e != cudaSuccess) return cuda_fail(e, "prim_to_cons launch");
    return FRSDG_OK;
}

int frsdg_rhs_host(frsdg_handle* h, double t, const double* U_host, double* rhs_host, void* stream)
{
    if (!h || !U_host || !rhs_host) return fail(FRSDG_ERR_ARG, "null argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    h->last = s;
    cudaError_t e;
    if (!h->d_stage)
    {
        e = cudaMalloc(&h->d_stage, sizeof(double) * 2 * h->ntot);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(staging)");
    }
    double* dU = h->d_stage;
    double* dR = h->d_stage + h->ntot;
    const int C = std::min(frsdg_handle::kHostChunks, h->Ny / 4);
    const bool chunked = h->cfg.dim == 2 && !h->win_rows && C >= 2;
    if (!chunked)
    {
        const size_t bytes = sizeof(double) * local_ntot(h);
        if ((e = cudaMemcpyAsync(dU, U_host, bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess)
            return cuda_fail(e, "H2D copy");
        int rc = run_residual(h, MODE_RHS, t, dU, nullptr, dR, stream);
        if (rc) return rc;
        if ((e = cudaMemcpyAsync(rhs_host, dR, bytes, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
            return cuda_fail(e, "D2H copy");
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "stream sync");
        return FRSDG_OK;
    }
    // 2D whole mesh: C row chunks (up to 32: 5.1e9 -> 5.7e9 DOF/s against 8 on the 1024^2
    // blast) through three streams -- upload chunk c, compute it once
    // its neighbour rows are there, download its rhs -- so that the host-to-device and
    // device-to-host transfers overlap each other and the kernels.  The chunks are the
    // kernel's row range on the whole arrays: the result is that of one launch.
    if (!h->hst[0])
    {
        for (cudaStream_t& q : h->hst)
            if ((e = cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking)) != cudaSuccess)
                return cuda_fail(e, "cudaStreamCreate");
        for (cudaEvent_t& ev : h->hev)
            if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess)
                return cuda_fail(e, "cudaEventCreate");
    }
    cudaEvent_t* up = h->hev;
    cudaEvent_t* done = h->hev + C;
    cudaEvent_t  start = h->hev[2 * C], finish = h->hev[2 * C + 1];
    const int64_t row = int64_t(h->Nx) * h->ndofs;  // doubles per element row
    auto r0 = [&](int c) { return c >= C ? h->Ny : int((int64_t(c) * h->Ny / C) & ~1); };
    const bool per_y = h->a2.per_y;
    if ((e = cudaEventRecord(start, s)) != cudaSuccess) return cuda_fail(e, "event record");
    for (cudaStream_t q : h->hst)
        if ((e = cudaStreamWaitEvent(q, start, 0)) != cudaSuccess) return cuda_fail(e, "stream wait");
    for (int c = 0; c < C; ++c)
    {
        const size_t bytes = sizeof(double) * size_t(row) * size_t(r0(c + 1) - r0(c));
        if ((e = cudaMemcpyAsync(dU + row * r0(c), U_host + row * r0(c), bytes, cudaMemcpyHostToDevice, h->hst[0])) !=
            cudaSuccess)
            return cuda_fail(e, "H2D copy");
        if ((e = cudaEventRecord(up[c], h->hst[0])) != cudaSuccess) return cuda_fail(e, "event record");
    }
    // a periodic mesh's first chunk reads the last row: compute it last
    for (int k = 0; k < C; ++k)
    {
        const int c = per_y ? (k + 1) % C : k;
        const int need[3] = {c, c + 1 < C ? c + 1 : (per_y ? 0 : c), c > 0 ? c - 1 : (per_y ? C - 1 : c)};
        for (int n : need)
            if ((e = cudaStreamWaitEvent(h->hst[1], up[n], 0)) != cudaSuccess) return cuda_fail(e, "stream wait");
        Fr2dArgs a = h->a2;
        a.t = t;
        a.mode = MODE_RHS;
        a.cond_sys = 0;
        a.U = dU;
        a.W = nullptr;
        a.out = dR;
        a.row_begin = r0(c);
        a.row_end = r0(c + 1);
        if ((e = dispatch2d<double>(h->n, h->cfg.gas_law, h->cfg.riemann, h->geo, a, h->hst[1])) != cudaSuccess)
            return cuda_fail(e, "residual launch");
        if ((e = cudaEventRecord(done[c], h->hst[1])) != cudaSuccess) return cuda_fail(e, "event record");
        if ((e = cudaStreamWaitEvent(h->hst[2], done[c], 0)) != cudaSuccess) return cuda_fail(e, "stream wait");
        const size_t bytes = sizeof(double) * size_t(row) * size_t(r0(c + 1) - r0(c));
        if ((e = cudaMemcpyAsync(rhs_host + row * r0(c), dR + row * r0(c), bytes, cudaMemcpyDeviceToHost, h->hst[2])) !=
            cudaSuccess)
            return cuda_fail(e, "D2H copy");
    }
    if ((e = cudaEventRecord(finish, h->hst[2])) != cudaSuccess) return cuda_fail(e, "event record");
    if ((e = cudaStreamWaitEvent(s, finish, 0)) != cudaSuccess) return cuda_fail(e, "stream wait");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "stream sync");
    return FRSDG_OK;
}

int frsdg_check_state(frsdg_handle* h, const double* U, void* stream)
{
    if (!h || !U) return fail(FRSDG_ERR_ARG, "null argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    h->last = s;
    const cudaError_t e = launch_check_density(h->cfg.dim, h->n, local_nelem(h), U, h->d_bad, s);
    if (e != cudaSuccess) return cuda_fail(e, "state-check launch");
    return FRSDG_OK;
}

int frsdg_device_math(int32_t op, const double* x, double* y, int64_t n, void* stream)
{
    if (op < 0 || op > 5 || n < 0 || (n > 0 && (!x || !y))) return fail(FRSDG_ERR_ARG, "bad argument");
    const cudaError_t e = launch_device_math(op, x, y, n, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "device-math launch");
    return FRSDG_OK;
}

int frsdg_tc_lines(int32_t n, const float* v, const double* D, float* out, int64_t lines, void* stream)
{
    if (n < 2 || n > 8 || lines < 0 || (lines > 0 && (!v || !D || !out))) return fail(FRSDG_ERR_ARG, "bad argument");
    if (lines == 0) return FRSDG_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int* err = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&err), sizeof(int), s);
    if (e != cudaSuccess) return cuda_fail(e, "tensor-core flag allocation");
    int h_err = 0;
    if ((e = cudaMemsetAsync(err, 0, sizeof(int), s)) == cudaSuccess &&
        (e = launch_tc_lines(n, v, D, out, lines, err, s)) == cudaSuccess)
        e = cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    const cudaError_t e2 = cudaFreeAsync(err, s);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "tensor-core line contraction");
    return h_err ? fail(FRSDG_ERR_CUDA, "tensor-core completion wait gave up") : FRSDG_OK;
}

int frsdg_status(frsdg_handle* h, int64_t* bad_nodes)
{
    if (!h || !bad_nodes) return fail(FRSDG_ERR_ARG, "null argument");
    unsigned long long v = 0;
    cudaError_t e = cudaStreamSynchronize(h->last);
    if (e != cudaSuccess) return cuda_fail(e, "status sync");
    e = cudaMemcpy(&v, h->d_bad, sizeof(v), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "status read");
    e = cudaMemset(h->d_bad, 0, sizeof(v));
    if (e != cudaSuccess) return cuda_fail(e, "status reset");
    *bad_nodes = int64_t(v);
    return FRSDG_OK;
}

} // extern "C"
