// residual1d.cuh -- FR residual of the 1D Euler equations.
//
// Reference: PhysicsEvaluator<Traits,1>::residual_kernel and local_steady_res,
// include/physics_impl_1D.hpp:9-94 and 124-181.  Each element solves the Riemann
// problems on both of its faces (as the reference does), builds
//   R[eq,i] = sum_j (2/dx) D(i,j) F_j  +  (2/dx) (dF_L dL(i) + dF_R dR(i)),
// and, for the radial coordinate system, adds the geometric source on the
// elements that are not physical-boundary elements.  Layout: element e at e*3n,
// value (eq, node) at eq*n + node.
#pragma once
#include "device_math.cuh"
#include "frsdg_internal.hpp"
#include "physics.cuh"

namespace frsdg
{

constexpr int kElems1D = 32; // elements per CTA

template <class S> struct NodeLoader1D;
template <> struct NodeLoader1D<double>
{
    __device__ static double load(const Fr1dArgs& a, int64_t idx) { return __ldg(a.U + idx); }
};
template <> struct NodeLoader1D<cplx>
{
    __device__ static cplx load(const Fr1dArgs& a, int64_t idx)
    {
        return cplx(__ldg(a.U + idx), __ldg(a.W + idx) * a.h);
    }
};

// prim_to_cons_elem (problem_def.hpp:36-51) for one 1D node in place.
template <class S> __device__ __forceinline__ void prim_to_cons1(S s[3])
{
    const S rho  = s_exp(s[0]);
    const S ssq  = S(0.0) + s[1] * s[1];
    const S rhoE = rho * (s_exp(s[2]) + S(0.5) * ssq);
    const S u    = s[1];
    s[0] = rho;
    s[1] = rho * u;
    s[2] = rhoE;
}

template <class S, int N, int GAS, int RIEM>
__global__ void __launch_bounds__(kThreads) fr1d_kernel(const Fr1dArgs a)
{
    constexpr int E  = kElems1D;
    constexpr int ND = 3 * N;
    __shared__ S sU[(E + 2) * ND];        // element slots -1..E
    __shared__ S sF[E * ND];
    __shared__ S sDL[E * 3], sDR[E * 3]; // F* - F at the left and right end of each element
    __shared__ double sD[N * N], sdL[N], sdR[N];

    const int tid = threadIdx.x;
    const int e0  = blockIdx.x * E;
    const int ne  = min(E, a.N - e0);
    for (int q = tid; q < N * N; q += kThreads) sD[q] = a.ops.D[q];
    for (int q = tid; q < N; q += kThreads) { sdL[q] = a.ops.dL[q]; sdR[q] = a.ops.dR[q]; }

    // load elements e0-1 .. e0+ne (periodic wrap; out-of-range slots unused)
    for (int q = tid; q < (ne + 2) * N; q += kThreads)
    {
        const int slot = q / N, node = q % N;
        int ge = e0 - 1 + slot;
        if (ge < 0) { if (!a.per) continue; ge += a.N; }
        if (ge >= a.N) { if (!a.per) continue; ge -= a.N; }
        S s[3];
        for (int eq = 0; eq < 3; ++eq) s[eq] = NodeLoader1D<S>::load(a, int64_t(ge) * ND + eq * N + node);
        if (a.cond_sys) prim_to_cons1(s);
        for (int eq = 0; eq < 3; ++eq) sU[slot * ND + eq * N + node] = s[eq];
    }
    __syncthreads();

    const GasParams g = a.gas;
    for (int q = tid; q < ne * N; q += kThreads)
    {
        const int e = q / N, node = q % N;
        const S* u = sU + (e + 1) * ND;
        S s[3] = {u[node], u[N + node], u[2 * N + node]};
        if (!density_ok(s_re(s[0])) && a.bad) atomicAdd(a.bad, 1ull);
        S F[3], p, rw, ee;
        flux1<GAS>(g, s, F, p, rw, ee);
        for (int eq = 0; eq < 3; ++eq) sF[e * ND + eq * N + node] = F[eq];
    }
    __syncthreads();

    // both faces of each element
    for (int q = tid; q < 2 * ne; q += kThreads)
    {
        const int e = q >> 1, side = q & 1, ge = e0 + e;
        const S* u = sU + (e + 1) * ND;
        S own[3], other[3];
        const int onode = side ? N - 1 : 0;
        for (int eq = 0; eq < 3; ++eq) own[eq] = u[eq * N + onode];
        const bool at_bc = !a.per && (side ? ge == a.N - 1 : ge == 0);
        if (at_bc)
        {
            const BcDev& b = a.bc[side];
            for (int eq = 0; eq < 3; ++eq) other[eq] = own[eq];
            if (b.kind == FRSDG_BC_WALL) other[1] = -own[1];
            else if (b.kind == FRSDG_BC_DIRICHLET)
                for (int eq = 0; eq < 3; ++eq) other[eq] = S(b.state[eq]);
        }
        else
        {
            const S* nb = sU + (e + (side ? 2 : 0)) * ND;
            const int nnode = side ? 0 : N - 1;
            for (int eq = 0; eq < 3; ++eq) other[eq] = nb[eq * N + nnode];
        }
        S Fs[3];
        if (side) riemann1<RIEM, GAS>(g, own, other, Fs);
        else riemann1<RIEM, GAS>(g, other, own, Fs);
        S* dst = side ? sDR : sDL;
        for (int eq = 0; eq < 3; ++eq) dst[e * 3 + eq] = Fs[eq] - sF[e * ND + eq * N + onode];
    }
    __syncthreads();

    for (int q = tid; q < ne * ND; q += kThreads)
    {
        const int e = q / ND, rem = q % ND, eq = rem / N, i = rem % N, ge = e0 + e;
        S r = S(0.0);
#pragma unroll
        for (int j = 0; j < N; ++j)
        {
            const double Dij = a.inv_jac * sD[i * N + j];
            r = r + Dij * sF[e * ND + eq * N + j];
        }
        r = r + a.inv_jac * (sDL[e * 3 + eq] * sdL[i] + sDR[e * 3 + eq] * sdR[i]);
        const bool boundary_elem = !a.per && (ge == 0 || ge == a.N - 1);
        if (a.radial && !boundary_elem)
        {
            // get_r (physics_evaluator.hpp:148-155) and the source of physics_impl_1D.hpp:70-90
            const S* u = sU + (e + 1) * ND;
            const S rho = u[i], rhoU = u[N + i], rhoE = u[2 * N + i];
            const S vel = rhoU / rho;
            const S pres = gas_pressure<GAS>(g, rho, rhoE / rho - S(0.5) * vel * vel);
            const double rad = (double(ge) + 0.5 * (a.ops.csi[i] + 1.0)) * a.h_elem;
            const double inv_r = (rad > 1e-8) ? 1.0 / rad : 0.0;
            const S src[3] = {inv_r * rhoU, inv_r * rhoU * vel, inv_r * vel * (rhoE + pres)};
            r = r + src[eq];
        }
        const int64_t gidx = int64_t(ge) * ND + rem;
        if constexpr (scalar_traits<S>::words == 2)
        {
            const S us = sU[(e + 1) * ND + rem];
            double jv  = a.sigma * s_im(us) * a.inv_h;
            jv += s_im(r) * a.inv_h;
            reinterpret_cast<double*>(a.out)[gidx] = jv;
        }
        else
        {
            store_residual(a.mode, a.W, a.st, reinterpret_cast<double*>(a.out), gidx, s_re(r));
        }
    }
}

template <class S, int N, int GAS, int RIEM> cudaError_t launch_fr1d_kernel(const Fr1dArgs& a, cudaStream_t st)
{
    dim3 grid((a.N + kElems1D - 1) / kElems1D);
    fr1d_kernel<S, N, GAS, RIEM><<<grid, kThreads, 0, st>>>(a);
    return cudaGetLastError();
}

template <class S, int N> cudaError_t launch_fr1d(int gas, int riem, const Fr1dArgs& a, cudaStream_t s)
{
    switch (gas * 2 + riem)
    {
        case 0: return launch_fr1d_kernel<S, N, 0, 0>(a, s);
        case 1: return launch_fr1d_kernel<S, N, 0, 1>(a, s);
        case 2: return launch_fr1d_kernel<S, N, 1, 0>(a, s);
        case 3: return launch_fr1d_kernel<S, N, 1, 1>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

} // namespace frsdg
