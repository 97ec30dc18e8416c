// stab.cu -- post-step stabilisation and the change of variables.
//
// PetscSolver::apply_stabilization -> limit_solution (petsc_solver_impl.hpp:683-702,
// physics_impl_2D.hpp:76-124, physics_impl_1D.hpp:96-121) with
// StabilizationTechniques::apply_element_stabilization (filter.hpp:716-755):
//   spectral filter only:  out = F u on every line;
//   WENO (+ shock sensor): WENO reconstruction on lines the sensor flags, copy
//                          elsewhere; with the filter also on, the reference
//                          overwrites every line with F u, so the filter result
//                          is what remains.
// In 2D each element gets 1/2 (x-line result + y-line result).  Neighbours across
// a non-periodic boundary are zero (the never-written ghost entries of a PETSc
// local vector).
#include "frsdg_internal.hpp"
#include "stab.hpp"

namespace frsdg
{

template <int N>
__device__ void stab_line(const StabArgs& a, const double* prev, const double* curr, const double* next,
                          double* out)
{
    if (!a.apply_filter && !a.apply_weno)
    {
        for (int i = 0; i < N; ++i) out[i] = curr[i];
        return;
    }
    if (a.apply_weno && !a.apply_filter)
    {
        // WENOLimiter::compute_smoothness (filter.hpp:586-616)
        auto smooth = [&](const double* v) {
            double cur[N], nxt[N];
            for (int i = 0; i < N; ++i) cur[i] = v[i];
            double beta = 0.0, factor = 4.0;
            for (int s = 1; s <= N - 1; ++s)
            {
                for (int r = 0; r < N; ++r)
                {
                    double acc = 0.0;
                    for (int c = 0; c < N; ++c) acc += a.D[r * N + c] * cur[c];
                    nxt[r] = acc;
                }
                double integ = 0.0;
                for (int i = 0; i < N; ++i)
                {
                    cur[i] = nxt[i];
                    integ += a.w[i] * cur[i] * cur[i];
                }
                beta += factor * (0.5 * integ);
                factor *= 4.0;
            }
            return beta;
        };
        const double b0 = smooth(prev), b1 = smooth(curr), b2 = smooth(next);
        // ShockSensor::detect_shock (filter.hpp:654-678)
        double cg0 = a.gam[0] / ((1.0e-6 + b0) * (1.0e-6 + b0));
        double cg1 = a.gam[1] / ((1.0e-6 + b1) * (1.0e-6 + b1));
        double cg2 = a.gam[2] / ((1.0e-6 + b2) * (1.0e-6 + b2));
        const double ws = cg0 + cg1 + cg2;
        cg0 /= ws; cg1 /= ws; cg2 /= ws;
        const double num = pow(fabs(cg0 / a.gam[0] - 1.0), a.theta) + pow(fabs(cg1 / a.gam[1] - 1.0), a.theta) +
                           pow(fabs(cg2 / a.gam[2] - 1.0), a.theta);
        const double r_j = num * a.one_over_norm;
        if (fabs(r_j) >= a.threshold)
        {
            // WENOLimiter::apply_weno_scalar (filter.hpp:519-544)
            double ap = 0.0, ac = 0.0, an = 0.0;
            for (int i = 0; i < N; ++i) { ap += a.w[i] * prev[i]; ac += a.w[i] * curr[i]; an += a.w[i] * next[i]; }
            ap *= 0.5; ac *= 0.5; an *= 0.5;
            for (int i = 0; i < N; ++i)
                out[i] = cg0 * (prev[i] - ap + ac) + cg1 * curr[i] + cg2 * (next[i] - an + ac);
            return;
        }
        for (int i = 0; i < N; ++i) out[i] = curr[i];
        return;
    }
    // SpectralFilter::apply_filter (filter.hpp:425-445)
    for (int r = 0; r < N; ++r)
    {
        double acc = 0.0;
        for (int c = 0; c < N; ++c) acc += a.F[r * N + c] * curr[c];
        out[r] = acc;
    }
}

template <int N> __global__ void __launch_bounds__(kThreads) stab2d_kernel(const StabArgs a)
{
    constexpr int NN = N * N, ND = 4 * NN, LPE = 8 * N; // lines per element
    constexpr int E = (kThreads / LPE) > 0 ? kThreads / LPE : 1;
    __shared__ double sX[E * ND], sY[E * ND];
    const int tid = threadIdx.x;
    const int64_t nel = int64_t(a.Nx) * a.Ny;
    const int64_t e0 = int64_t(blockIdx.x) * E;
    const int le = tid / LPE, line = tid % LPE;
    const int64_t ge = e0 + le;
    const bool active = le < E && ge < nel;
    if (active)
    {
        const int gi = int(ge % a.Nx), gj = int(ge / a.Nx);
        const bool xdir = line < 4 * N;
        const int eq = (line % (4 * N)) / N, m = line % N;
        auto elem = [&](int i, int j) -> const double* {
            if (i < 0 || i >= a.Nx) { if (!a.per_x) return nullptr; i = (i + a.Nx) % a.Nx; }
            if (j < 0 || j >= a.Ny) { if (!a.per_y) return nullptr; j = (j + a.Ny) % a.Ny; }
            return a.src + (int64_t(j) * a.Nx + i) * ND;
        };
        const double* pC = elem(gi, gj);
        const double* pP = xdir ? elem(gi - 1, gj) : elem(gi, gj - 1);
        const double* pN = xdir ? elem(gi + 1, gj) : elem(gi, gj + 1);
        double pv[N], cv[N], nv[N], o[N];
        for (int t = 0; t < N; ++t)
        {
            const int node = xdir ? (m * N + t) : (t * N + m);
            cv[t] = pC[node * 4 + eq];
            pv[t] = (a.apply_weno && pP) ? pP[node * 4 + eq] : 0.0;
            nv[t] = (a.apply_weno && pN) ? pN[node * 4 + eq] : 0.0;
        }
        stab_line<N>(a, pv, cv, nv, o);
        double* dst = xdir ? sX : sY;
        for (int t = 0; t < N; ++t)
        {
            const int node = xdir ? (m * N + t) : (t * N + m);
            dst[le * ND + node * 4 + eq] = o[t];
        }
    }
    __syncthreads();
    for (int q = tid; q < E * ND; q += kThreads)
    {
        const int l2 = q / ND;
        const int64_t g2 = e0 + l2;
        if (g2 < nel) a.dst[g2 * ND + (q % ND)] = 0.5 * (sX[q] + sY[q]);
    }
}

template <int N> __global__ void __launch_bounds__(kThreads) stab1d_kernel(const StabArgs a)
{
    constexpr int ND = 3 * N;
    const int64_t q = int64_t(blockIdx.x) * kThreads + threadIdx.x;
    if (q >= int64_t(a.Nx) * 3) return;
    const int e = int(q / 3), eq = int(q % 3);
    auto elem = [&](int i) -> const double* {
        if (i < 0 || i >= a.Nx) { if (!a.per_x) return nullptr; i = (i + a.Nx) % a.Nx; }
        return a.src + int64_t(i) * ND;
    };
    const double* pC = elem(e);
    const double* pP = elem(e - 1);
    const double* pN = elem(e + 1);
    double pv[N], cv[N], nv[N], o[N];
    for (int t = 0; t < N; ++t)
    {
        cv[t] = pC[eq * N + t];
        pv[t] = (a.apply_weno && pP) ? pP[eq * N + t] : 0.0;
        nv[t] = (a.apply_weno && pN) ? pN[eq * N + t] : 0.0;
    }
    stab_line<N>(a, pv, cv, nv, o);
    for (int t = 0; t < N; ++t) a.dst[int64_t(e) * ND + eq * N + t] = o[t];
}

// prim_to_cons_elem (problem_def.hpp:286-301) on every node.
__global__ void prim_to_cons2d_kernel(const double* __restrict__ in, double* __restrict__ out, int64_t nodes)
{
    const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= nodes) return;
    const double2 a0 = reinterpret_cast<const double2*>(in)[2 * q];
    const double2 a1 = reinterpret_cast<const double2*>(in)[2 * q + 1];
    const double rho  = exp(a0.x);
    const double ssq  = (0.0 + a0.y * a0.y) + a1.x * a1.x;
    const double rhoE = rho * (exp(a1.y) + 0.5 * ssq);
    reinterpret_cast<double2*>(out)[2 * q]     = make_double2(rho, rho * a0.y);
    reinterpret_cast<double2*>(out)[2 * q + 1] = make_double2(rho * a1.x, rhoE);
}

__global__ void prim_to_cons1d_kernel(const double* __restrict__ in, double* __restrict__ out, int64_t nelem, int n)
{
    const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= nelem * n) return;
    const int64_t e = q / n;
    const int     k = int(q % n);
    const double* p = in + e * 3 * n;
    double*       c = out + e * 3 * n;
    const double rho = exp(p[k]), vel = p[n + k], ie = p[2 * n + k];
    const double ssq = 0.0 + vel * vel;
    c[k]         = rho;
    c[n + k]     = rho * vel;
    c[2 * n + k] = rho * (exp(ie) + 0.5 * ssq);
}

template <int N> cudaError_t launch_stab_n(const StabArgs& a, cudaStream_t s)
{
    if (a.dim == 2)
    {
        constexpr int LPE = 8 * N;
        constexpr int E = (kThreads / LPE) > 0 ? kThreads / LPE : 1;
        const int64_t nel = int64_t(a.Nx) * a.Ny;
        stab2d_kernel<N><<<unsigned((nel + E - 1) / E), kThreads, 0, s>>>(a);
    }
    else
    {
        const int64_t lines = int64_t(a.Nx) * 3;
        stab1d_kernel<N><<<unsigned((lines + kThreads - 1) / kThreads), kThreads, 0, s>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t launch_stab(int n, const StabArgs& a, cudaStream_t s)
{
    switch (n)
    {
        case 2: return launch_stab_n<2>(a, s);
        case 3: return launch_stab_n<3>(a, s);
        case 4: return launch_stab_n<4>(a, s);
        case 5: return launch_stab_n<5>(a, s);
        case 6: return launch_stab_n<6>(a, s);
        case 7: return launch_stab_n<7>(a, s);
        case 8: return launch_stab_n<8>(a, s);
        case 9: return launch_stab_n<9>(a, s);
        case 10: return launch_stab_n<10>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_prim_to_cons(int dim, int n, int64_t nelem, const double* in, double* out, cudaStream_t s)
{
    if (dim == 2)
    {
        const int64_t nodes = nelem * n * n;
        prim_to_cons2d_kernel<<<unsigned((nodes + 255) / 256), 256, 0, s>>>(in, out, nodes);
    }
    else
    {
        const int64_t nodes = nelem * n;
        prim_to_cons1d_kernel<<<unsigned((nodes + 255) / 256), 256, 0, s>>>(in, out, nelem, n);
    }
    return cudaGetLastError();
}

} // namespace frsdg
