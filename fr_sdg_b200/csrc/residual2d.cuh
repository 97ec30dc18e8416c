// residual2d.cuh -- fused FR residual of the 2D Euler equations.
//
// One CTA owns a tile of TX x TY elements and does, in one pass over HBM:
//   1. load the tile's states (DMDA natural order, node-major AoS) and the four
//      halo traces of its neighbours into shared memory (with the complex-step
//      seed u + i h v and the prim->cons map applied on the fly when asked);
//   2. Euler fluxes F, G of every node (euler_fluxes_2d_w_p);
//   3. one Riemann solve per face point of the tile, on faces interior to the
//      tile and on its four edges, with boundary ghosts on physical edges; the
//      jumps scale*(F* - F.n) of each adjacent element go to shared memory;
//   4. per (node, equation) the chain-rule volume term of compute_volume_term
//      plus the four VCJH lifts, then the output form (R, -R, U_t + R or the
//      complex-step JVP) written once, coalesced.
// Reference: PhysicsEvaluator<Traits,2>::residual_kernel and compute_volume_term,
// include/physics_impl_2D.hpp:268-357 and 646-902, summed in the same order
// (volume, left x-face, right x-face, bottom y-face, top y-face).
#pragma once
#include "device_math.cuh"
#include "frsdg_internal.hpp"
#include "physics.cuh"

namespace frsdg
{

template <class S, int N> struct Tile2D
{
    static constexpr int TX = tile_x(N);
    static constexpr int TY = tile_y(N);
    static constexpr int NN = N * N;
    static constexpr int TE = TX * TY;
    // offsets in units of S
    static constexpr int oU   = 0;
    static constexpr int oHXL = oU + TE * NN * 4;
    static constexpr int oHXR = oHXL + TY * N * 4;
    static constexpr int oHYB = oHXR + TY * N * 4;
    static constexpr int oHYT = oHYB + TX * N * 4;
    static constexpr int oF   = oHYT + TX * N * 4;
    static constexpr int oG   = oF + 4 * TE * NN;
    static constexpr int oDXL = oG + 4 * TE * NN;
    static constexpr int oDXR = oDXL + TE * 4 * N;
    static constexpr int oDYB = oDXR + TE * 4 * N;
    static constexpr int oDYT = oDYB + TE * 4 * N;
    static constexpr int nS   = oDYT + TE * 4 * N;
    static constexpr size_t bytes = size_t(nS) * sizeof(S) + sizeof(double) * (NN + 2 * N);
};

// Load one node's 4 values from the input vectors and form the scalar the residual
// works on: the state itself, M(prim) for the change of variables, or the
// complex-step point M(u + i h v).
template <class S> struct NodeLoader;

template <> struct NodeLoader<double>
{
    __device__ static void load(const Fr2dArgs& a, int64_t off, double s[4])
    {
        const double2 x0 = __ldg(reinterpret_cast<const double2*>(a.U + off));
        const double2 x1 = __ldg(reinterpret_cast<const double2*>(a.U + off + 2));
        s[0] = x0.x; s[1] = x0.y; s[2] = x1.x; s[3] = x1.y;
        if (a.cond_sys)
        {
            // prim_to_cons_elem (problem_def.hpp:286-301)
            const double rho  = exp(s[0]);
            const double ssq  = (0.0 + s[1] * s[1]) + s[2] * s[2];
            const double rhoE = rho * (exp(s[3]) + 0.5 * ssq);
            const double u = s[1], v = s[2];
            s[0] = rho; s[1] = rho * u; s[2] = rho * v; s[3] = rhoE;
        }
    }
};

template <> struct NodeLoader<float>
{
    __device__ static void load(const Fr2dArgs& a, int64_t off, float s[4])
    {
        const double2 x0 = __ldg(reinterpret_cast<const double2*>(a.U + off));
        const double2 x1 = __ldg(reinterpret_cast<const double2*>(a.U + off + 2));
        s[0] = float(x0.x); s[1] = float(x0.y); s[2] = float(x1.x); s[3] = float(x1.y);
    }
};

template <> struct NodeLoader<cplx>
{
    __device__ static void load(const Fr2dArgs& a, int64_t off, cplx s[4])
    {
        const double2 x0 = __ldg(reinterpret_cast<const double2*>(a.U + off));
        const double2 x1 = __ldg(reinterpret_cast<const double2*>(a.U + off + 2));
        const double2 v0 = __ldg(reinterpret_cast<const double2*>(a.W + off));
        const double2 v1 = __ldg(reinterpret_cast<const double2*>(a.W + off + 2));
        s[0] = cplx(x0.x, v0.x * a.h);
        s[1] = cplx(x0.y, v0.y * a.h);
        s[2] = cplx(x1.x, v1.x * a.h);
        s[3] = cplx(x1.y, v1.y * a.h);
        if (a.cond_sys)
        {
            const cplx rho  = s_exp(s[0]);
            const cplx ssq  = (cplx(0.0) + s[1] * s[1]) + s[2] * s[2];
            const cplx rhoE = rho * (s_exp(s[3]) + 0.5 * ssq);
            const cplx u = s[1], v = s[2];
            s[0] = rho; s[1] = rho * u; s[2] = rho * v; s[3] = rhoE;
        }
    }
};

template <class S> __device__ __forceinline__ void store_out(void* out, int64_t idx, S r, const Fr2dArgs& a,
                                                             const S& u_self);

template <>
__device__ __forceinline__ void store_out<double>(void* out, int64_t idx, double r, const Fr2dArgs& a,
                                                  const double&)
{
    double v;
    if (a.mode == MODE_RHS) v = -r;
    else if (a.mode == MODE_IFUNC) v = __ldg(a.W + idx) + r;
    else v = r;
    reinterpret_cast<double*>(out)[idx] = v;
}
template <>
__device__ __forceinline__ void store_out<float>(void* out, int64_t idx, float r, const Fr2dArgs& a, const float&)
{
    reinterpret_cast<float*>(out)[idx] = (a.mode == MODE_RHS) ? -r : r;
}
template <>
__device__ __forceinline__ void store_out<cplx>(void* out, int64_t idx, cplx r, const Fr2dArgs& a,
                                                const cplx& u_self)
{
    double jv = a.sigma * u_self.im * a.inv_h;
    jv += r.im * a.inv_h;
    reinterpret_cast<double*>(out)[idx] = jv;
}

template <class S, int N, int GAS, int RIEM, int GEO>
__global__ void __launch_bounds__(kThreads) fr2d_kernel(const Fr2dArgs a)
{
    using T = Tile2D<S, N>;
    constexpr int TX = T::TX, TY = T::TY, NN = T::NN;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    S*      sm  = reinterpret_cast<S*>(smem_raw);
    double* sD  = reinterpret_cast<double*>(smem_raw + size_t(T::nS) * sizeof(S));
    double* sdL = sD + NN;
    double* sdR = sdL + N;
    S* sU  = sm + T::oU;
    S* sHXL = sm + T::oHXL;
    S* sHXR = sm + T::oHXR;
    S* sHYB = sm + T::oHYB;
    S* sHYT = sm + T::oHYT;
    S* sF  = sm + T::oF;
    S* sG  = sm + T::oG;
    S* sDXL = sm + T::oDXL;
    S* sDXR = sm + T::oDXR;
    S* sDYB = sm + T::oDYB;
    S* sDYT = sm + T::oDYT;

    const int tid = threadIdx.x;
    const int Nx = a.Nx, Ny = a.Ny;
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
    const int txe = min(TX, Nx - i0), tye = min(TY, Ny - j0);
    constexpr int ND = 4 * NN; // doubles per element

    for (int q = tid; q < NN; q += kThreads) sD[q] = a.ops.D[q];
    for (int q = tid; q < N; q += kThreads) { sdL[q] = a.ops.dL[q]; sdR[q] = a.ops.dR[q]; }

    // ---- 1. load tile and halo traces
    for (int q = tid; q < TY * TX * NN; q += kThreads)
    {
        const int ty = q / (TX * NN), rem = q % (TX * NN), tx = rem / NN, node = rem % NN;
        if (ty < tye && tx < txe)
        {
            const int64_t off = (int64_t(j0 + ty) * Nx + (i0 + tx)) * ND + node * 4;
            S s[4];
            NodeLoader<S>::load(a, off, s);
            S* d = sU + ((ty * TX + tx) * NN + node) * 4;
            d[0] = s[0]; d[1] = s[1]; d[2] = s[2]; d[3] = s[3];
        }
    }
    for (int q = tid; q < 2 * TY * N + 2 * TX * N; q += kThreads)
    {
        int     side, r, m;
        int     ge_i = -1, ge_j = -1, node = 0;
        S*      dst;
        if (q < 2 * TY * N)
        {
            side = q / (TY * N); r = (q % (TY * N)) / N; m = q % N;
            if (r >= tye) continue;
            ge_j = j0 + r;
            if (side == 0) { ge_i = i0 - 1; if (ge_i < 0) { if (!a.per_x) continue; ge_i += Nx; } node = m * N + (N - 1); dst = sHXL + (r * N + m) * 4; }
            else { ge_i = i0 + txe; if (ge_i >= Nx) { if (!a.per_x) continue; ge_i -= Nx; } node = m * N; dst = sHXR + (r * N + m) * 4; }
        }
        else
        {
            const int qq = q - 2 * TY * N;
            side = qq / (TX * N); r = (qq % (TX * N)) / N; m = qq % N;
            if (r >= txe) continue;
            ge_i = i0 + r;
            if (side == 0) { ge_j = j0 - 1; if (ge_j < 0) { if (!a.per_y) continue; ge_j += Ny; } node = (N - 1) * N + m; dst = sHYB + (r * N + m) * 4; }
            else { ge_j = j0 + tye; if (ge_j >= Ny) { if (!a.per_y) continue; ge_j -= Ny; } node = m; dst = sHYT + (r * N + m) * 4; }
        }
        const int64_t off = (int64_t(ge_j) * Nx + ge_i) * ND + node * 4;
        S s[4];
        NodeLoader<S>::load(a, off, s);
        dst[0] = s[0]; dst[1] = s[1]; dst[2] = s[2]; dst[3] = s[3];
    }
    __syncthreads();

    // ---- 2. volume fluxes
    const GasParams g = a.gas;
    for (int q = tid; q < TY * TX * NN; q += kThreads)
    {
        const int e = q / NN, node = q % NN;
        const int ty = e / TX, tx = e % TX;
        if (ty < tye && tx < txe)
        {
            const S* u = sU + q * 4;
            S s[4] = {u[0], u[1], u[2], u[3]};
            if (!(s_re(s[0]) > 0.0) && a.bad) atomicAdd(a.bad, 1ull);
            const Prim2<S> pr = prim2<GAS>(g, s);
            S F[4], G[4];
            fluxes2(s, pr, F, G);
#pragma unroll
            for (int eq = 0; eq < 4; ++eq)
            {
                sF[(eq * T::TE + e) * NN + node] = F[eq];
                sG[(eq * T::TE + e) * NN + node] = G[eq];
            }
        }
    }
    __syncthreads();

    // ---- 3. faces
    const int nxf = (txe + 1) * tye * N;
    const int nyf = txe * (tye + 1) * N;
    for (int q = tid; q < nxf + nyf; q += kThreads)
    {
        S UA[4], UB[4];
        double nx, ny;
        if (q < nxf)
        {
            // x-face I (0..txe) of tile row ty, face point l
            const int l = q % N, r = q / N, I = r % (txe + 1), ty = r / (txe + 1);
            const int gI = i0 + I, gj = j0 + ty;
            if constexpr (GEO == GEO_CURVED)
            {
                const double2 nn = __ldg(reinterpret_cast<const double2*>(a.xnorm) + (int64_t(gj) * (Nx + 1) + gI) * N + l);
                nx = nn.x; ny = nn.y;
            }
            else { nx = 1.0; ny = 0.0; }
            const bool inL = I > 0, inR = I < txe;
            const bool bcL = !inL && gI == 0 && !a.per_x;
            const bool bcR = !inR && gI == Nx && !a.per_x;
            const S* pL = inL ? sU + ((ty * TX + I - 1) * NN + l * N + (N - 1)) * 4 : sHXL + (ty * N + l) * 4;
            const S* pR = inR ? sU + ((ty * TX + I) * NN + l * N) * 4 : sHXR + (ty * N + l) * 4;
            if (!bcL) { UA[0] = pL[0]; UA[1] = pL[1]; UA[2] = pL[2]; UA[3] = pL[3]; }
            if (!bcR) { UB[0] = pR[0]; UB[1] = pR[1]; UB[2] = pR[2]; UB[3] = pR[3]; }
            if (bcL)
            {
                const double2 xy = __ldg(reinterpret_cast<const double2*>(a.bxy[FRSDG_LEFT]) + gj * N + l);
                bc_ghost2<GAS>(a.bc[FRSDG_LEFT], FRSDG_LEFT, g, a.t, xy.x, xy.y, nx, ny, a.Lx, a.Ly, UB, UA);
            }
            if (bcR)
            {
                const double2 xy = __ldg(reinterpret_cast<const double2*>(a.bxy[FRSDG_RIGHT]) + gj * N + l);
                bc_ghost2<GAS>(a.bc[FRSDG_RIGHT], FRSDG_RIGHT, g, a.t, xy.x, xy.y, nx, ny, a.Lx, a.Ly, UA, UB);
            }
            S Fs[4];
            riemann2<RIEM, GAS>(g, UA, UB, nx, ny, Fs);
            if (inL)
            {
                const int e = ty * TX + I - 1, node = l * N + (N - 1);
                double sc;
                if constexpr (GEO == GEO_CURVED)
                {
                    const double2 m = __ldg(reinterpret_cast<const double2*>(a.metrics + ((int64_t(gj) * Nx + gI - 1) * NN + node) * 4));
                    sc = sqrt(m.x * m.x + m.y * m.y);
                }
                else sc = a.scale_x;
#pragma unroll
                for (int eq = 0; eq < 4; ++eq)
                {
                    const S fn = sF[(eq * T::TE + e) * NN + node] * nx + sG[(eq * T::TE + e) * NN + node] * ny;
                    sDXR[(e * 4 + eq) * N + l] = sc * (Fs[eq] - fn);
                }
            }
            if (inR)
            {
                const int e = ty * TX + I, node = l * N;
                double sc;
                if constexpr (GEO == GEO_CURVED)
                {
                    const double2 m = __ldg(reinterpret_cast<const double2*>(a.metrics + ((int64_t(gj) * Nx + gI) * NN + node) * 4));
                    sc = sqrt(m.x * m.x + m.y * m.y);
                }
                else sc = a.scale_x;
#pragma unroll
                for (int eq = 0; eq < 4; ++eq)
                {
                    const S fn = sF[(eq * T::TE + e) * NN + node] * nx + sG[(eq * T::TE + e) * NN + node] * ny;
                    sDXL[(e * 4 + eq) * N + l] = sc * (Fs[eq] - fn);
                }
            }
        }
        else
        {
            // y-face J (0..tye) of tile column tx, face point k
            const int qq = q - nxf;
            const int k = qq % N, r = qq / N, tx = r % txe, J = r / txe;
            const int gi = i0 + tx, gJ = j0 + J;
            if constexpr (GEO == GEO_CURVED)
            {
                const double2 nn = __ldg(reinterpret_cast<const double2*>(a.ynorm) + (int64_t(gJ) * Nx + gi) * N + k);
                nx = nn.x; ny = nn.y;
            }
            else { nx = 0.0; ny = 1.0; }
            const bool inB = J > 0, inT = J < tye;
            const bool bcB = !inB && gJ == 0 && !a.per_y;
            const bool bcT = !inT && gJ == Ny && !a.per_y;
            const S* pB = inB ? sU + (((J - 1) * TX + tx) * NN + (N - 1) * N + k) * 4 : sHYB + (tx * N + k) * 4;
            const S* pT = inT ? sU + ((J * TX + tx) * NN + k) * 4 : sHYT + (tx * N + k) * 4;
            if (!bcB) { UA[0] = pB[0]; UA[1] = pB[1]; UA[2] = pB[2]; UA[3] = pB[3]; }
            if (!bcT) { UB[0] = pT[0]; UB[1] = pT[1]; UB[2] = pT[2]; UB[3] = pT[3]; }
            if (bcB)
            {
                const double2 xy = __ldg(reinterpret_cast<const double2*>(a.bxy[FRSDG_BOTTOM]) + gi * N + k);
                bc_ghost2<GAS>(a.bc[FRSDG_BOTTOM], FRSDG_BOTTOM, g, a.t, xy.x, xy.y, nx, ny, a.Lx, a.Ly, UB, UA);
            }
            if (bcT)
            {
                const double2 xy = __ldg(reinterpret_cast<const double2*>(a.bxy[FRSDG_TOP]) + gi * N + k);
                bc_ghost2<GAS>(a.bc[FRSDG_TOP], FRSDG_TOP, g, a.t, xy.x, xy.y, nx, ny, a.Lx, a.Ly, UA, UB);
            }
            S Fs[4];
            riemann2<RIEM, GAS>(g, UA, UB, nx, ny, Fs);
            if (inB)
            {
                const int e = (J - 1) * TX + tx, node = (N - 1) * N + k;
                double sc;
                if constexpr (GEO == GEO_CURVED)
                {
                    const double2 m = __ldg(reinterpret_cast<const double2*>(a.metrics + ((int64_t(gJ - 1) * Nx + gi) * NN + node) * 4) + 1);
                    sc = sqrt(m.x * m.x + m.y * m.y);
                }
                else sc = a.scale_y;
#pragma unroll
                for (int eq = 0; eq < 4; ++eq)
                {
                    const S fn = sF[(eq * T::TE + e) * NN + node] * nx + sG[(eq * T::TE + e) * NN + node] * ny;
                    sDYT[(e * 4 + eq) * N + k] = sc * (Fs[eq] - fn);
                }
            }
            if (inT)
            {
                const int e = J * TX + tx, node = k;
                double sc;
                if constexpr (GEO == GEO_CURVED)
                {
                    const double2 m = __ldg(reinterpret_cast<const double2*>(a.metrics + ((int64_t(gJ) * Nx + gi) * NN + node) * 4) + 1);
                    sc = sqrt(m.x * m.x + m.y * m.y);
                }
                else sc = a.scale_y;
#pragma unroll
                for (int eq = 0; eq < 4; ++eq)
                {
                    const S fn = sF[(eq * T::TE + e) * NN + node] * nx + sG[(eq * T::TE + e) * NN + node] * ny;
                    sDYB[(e * 4 + eq) * N + k] = sc * (Fs[eq] - fn);
                }
            }
        }
    }
    __syncthreads();

    // ---- 4. volume term + lifts, output
    for (int q = tid; q < TY * TX * ND; q += kThreads)
    {
        const int e = q / ND, rem = q % ND, node = rem >> 2, eq = rem & 3;
        const int ty = e / TX, tx = e % TX;
        if (ty >= tye || tx >= txe) continue;
        const int k = node % N, l = node / N;
        const S* Fe = sF + (eq * T::TE + e) * NN;
        const S* Ge = sG + (eq * T::TE + e) * NN;
        S dF_dxi = S(0.0), dG_deta = S(0.0);
        S dG_dxi = S(0.0), dF_deta = S(0.0);
#pragma unroll
        for (int m = 0; m < N; ++m)
        {
            if constexpr (GEO == GEO_CURVED) dG_dxi = dG_dxi + sD[k * N + m] * Ge[l * N + m];
            dF_dxi = dF_dxi + sD[k * N + m] * Fe[l * N + m];
        }
#pragma unroll
        for (int m = 0; m < N; ++m)
        {
            dG_deta = dG_deta + sD[l * N + m] * Ge[m * N + k];
            if constexpr (GEO == GEO_CURVED) dF_deta = dF_deta + sD[l * N + m] * Fe[m * N + k];
        }
        const int64_t gidx = (int64_t(j0 + ty) * Nx + (i0 + tx)) * ND + rem;
        S R;
        if constexpr (GEO == GEO_CURVED)
        {
            const double* mt = a.metrics + (int64_t(j0 + ty) * Nx + (i0 + tx)) * ND + node * 4;
            const double2 m0 = __ldg(reinterpret_cast<const double2*>(mt));
            const double2 m1 = __ldg(reinterpret_cast<const double2*>(mt) + 1);
            const S px = m0.x * dF_dxi + m1.x * dF_deta;
            const S py = m0.y * dG_dxi + m1.y * dG_deta;
            R = px + py;
        }
        else
        {
            const S px = a.xi_x * dF_dxi;
            const S py = a.eta_y * dG_deta;
            R = px + py;
        }
        R = R + sDXL[(e * 4 + eq) * N + l] * sdL[k];
        R = R + sDXR[(e * 4 + eq) * N + l] * sdR[k];
        R = R + sDYB[(e * 4 + eq) * N + k] * sdL[l];
        R = R + sDYT[(e * 4 + eq) * N + k] * sdR[l];
        store_out<S>(a.out, gidx, R, a, sU[(e * NN + node) * 4 + eq]);
    }
}

template <class S, int N, int GAS, int RIEM, int GEO>
cudaError_t launch_fr2d_kernel(const Fr2dArgs& a, cudaStream_t st)
{
    using T = Tile2D<S, N>;
    auto kern = fr2d_kernel<S, N, GAS, RIEM, GEO>;
    static bool attr_done = false;
    if (!attr_done)
    {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(T::bytes));
        if (e != cudaSuccess) return e;
        attr_done = true;
    }
    dim3 grid((a.Nx + T::TX - 1) / T::TX, (a.Ny + T::TY - 1) / T::TY);
    kern<<<grid, kThreads, T::bytes, st>>>(a);
    return cudaGetLastError();
}

template <class S, int N> cudaError_t launch_fr2d(int gas, int riem, int geo, const Fr2dArgs& a, cudaStream_t s)
{
    const int key = gas * 4 + riem * 2 + geo;
    switch (key)
    {
        case 0: return launch_fr2d_kernel<S, N, 0, 0, 0>(a, s);
        case 1: return launch_fr2d_kernel<S, N, 0, 0, 1>(a, s);
        case 2: return launch_fr2d_kernel<S, N, 0, 1, 0>(a, s);
        case 3: return launch_fr2d_kernel<S, N, 0, 1, 1>(a, s);
        case 4: return launch_fr2d_kernel<S, N, 1, 0, 0>(a, s);
        case 5: return launch_fr2d_kernel<S, N, 1, 0, 1>(a, s);
        case 6: return launch_fr2d_kernel<S, N, 1, 1, 0>(a, s);
        case 7: return launch_fr2d_kernel<S, N, 1, 1, 1>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

} // namespace frsdg
