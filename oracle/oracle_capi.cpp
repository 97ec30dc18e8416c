// oracle_capi.cpp -- extern "C" wrapper of the CPU oracle for ctypes.
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py as the checker; the product library never links it.
#include "frsdg_oracle.hpp"

#include <cstring>
#include <exception>
#include <string>

using namespace frsdg_oracle;

namespace
{
thread_local std::string g_err;
template <class F> int guarded(F&& f)
{
    try
    {
        f();
        return 0;
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return -1;
    }
}
} // namespace

extern "C" {

const char* oracle_last_error() { return g_err.c_str(); }

void* oracle_create(const frsdg_config* cfg)
{
    try
    {
        return new Problem(*cfg);
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return nullptr;
    }
}

void oracle_destroy(void* h) { delete static_cast<Problem*>(h); }

void oracle_set_threads(void* h, int n) { static_cast<Problem*>(h)->nthreads = n > 0 ? n : 1; }

int64_t oracle_n_dofs(void* h) { return static_cast<Problem*>(h)->n_total(); }

int oracle_residual(void* h, double t, const double* U, double* R)
{
    return guarded([&] { residual(*static_cast<Problem*>(h), t, U, R); });
}

// Complex residual on interleaved (re, im) arrays; used to check the complex path.
int oracle_residual_complex(void* h, double t, const double* U, double* R)
{
    return guarded([&] {
        residual(*static_cast<Problem*>(h), t, reinterpret_cast<const cplx*>(U), reinterpret_cast<cplx*>(R));
    });
}

int oracle_rhs(void* h, double t, const double* U, double* F)
{
    return guarded([&] { rhs(*static_cast<Problem*>(h), t, U, F); });
}

int oracle_ifunction(void* h, double t, const double* U, const double* Udot, double* F)
{
    return guarded([&] { ifunction(*static_cast<Problem*>(h), t, U, Udot, F); });
}

int oracle_jvp(void* h, double t, double sigma, const double* U, const double* V, double* JV)
{
    return guarded([&] { jvp(*static_cast<Problem*>(h), t, sigma, U, V, JV); });
}

int oracle_post_step(void* h, double* U)
{
    return guarded([&] { post_step_full(*static_cast<Problem*>(h), U); });
}

// The positivity limiter alone (applied to every Runge-Kutta stage).
int oracle_pp_limit(void* h, double* U)
{
    return guarded([&] { pp_limit(*static_cast<Problem*>(h), U); });
}

int oracle_prim_to_cons(void* h, const double* prim, double* cons)
{
    return guarded([&] { prim_to_cons(*static_cast<Problem*>(h), prim, cons); });
}

int oracle_reference_element(int p, double c, double* nodes, double* w, double* D, double* dL, double* dR)
{
    return guarded([&] {
        const auto r = make_ref_element(p, c);
        std::memcpy(nodes, r.csi.data(), sizeof(double) * r.n);
        std::memcpy(w, r.w.data(), sizeof(double) * r.n);
        std::memcpy(D, r.D.data(), sizeof(double) * r.n * r.n);
        std::memcpy(dL, r.dL.data(), sizeof(double) * r.n);
        std::memcpy(dR, r.dR.data(), sizeof(double) * r.n);
    });
}

int oracle_filter_matrix(int p, int cut_off, int strength, double alpha, double* F)
{
    return guarded([&] {
        const auto r = make_ref_element(p, 0.0);
        const auto f = make_filter_matrix(r, cut_off, strength, alpha);
        std::memcpy(F, f.data(), sizeof(double) * r.n * r.n);
    });
}

// Per-node composite metrics (xi_x, xi_y, eta_x, eta_y, detJ) in DMDA element
// order [elem][node l*n+k][5]; used by tests to check cached geometry.
int oracle_node_metrics(void* h, double* out)
{
    return guarded([&] {
        const Problem& P = *static_cast<Problem*>(h);
        for (int j = 0; j < P.Ny; ++j)
            for (int i = 0; i < P.Nx; ++i)
                for (int l = 0; l < P.n; ++l)
                    for (int k = 0; k < P.n; ++k)
                    {
                        const auto m = P.metrics(P.comp_x(i, k), P.comp_y(j, l));
                        double* o = out + (((int64_t(j) * P.Nx + i) * P.n + l) * P.n + k) * 5;
                        o[0] = m.xi_x; o[1] = m.xi_y; o[2] = m.eta_x; o[3] = m.eta_y; o[4] = m.detJ;
                    }
    });
}

// Physical coordinates of every node, [elem][node][2].
int oracle_node_coords(void* h, double* out)
{
    return guarded([&] {
        const Problem& P = *static_cast<Problem*>(h);
        for (int j = 0; j < P.Ny; ++j)
            for (int i = 0; i < P.Nx; ++i)
                for (int l = 0; l < P.n; ++l)
                    for (int k = 0; k < P.n; ++k)
                    {
                        const auto xy = P.geom.coords(P.comp_x(i, k), P.comp_y(j, l));
                        double* o = out + (((int64_t(j) * P.Nx + i) * P.n + l) * P.n + k) * 2;
                        o[0] = xy.first; o[1] = xy.second;
                    }
    });
}

} // extern "C"
