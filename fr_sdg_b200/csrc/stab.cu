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
#include "device_math.cuh"
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

// ---- 2D: tiles of elements staged in shared memory -------------------------
// One CTA owns TX x TY elements.  It loads them, and for WENO the face neighbours
// across the tile edges (left/right columns, bottom/top rows), into shared memory
// with coalesced copies of whole elements; computes the smoothness indicator of
// every line once (tile lines in both directions, halo lines in the direction that
// crosses the tile edge), so each line's indicator serves the line itself and its
// two neighbours; then limits each tile line and combines the x- and y-line results
// per node, and stores the tile with coalesced writes.
template <int N> struct StabTile
{
    static constexpr int TX = N <= 6 ? 4 : 2, TY = TX;
    static constexpr int TE = TX * TY, NN = N * N, ND = 4 * NN;
    static constexpr int NSLOT = TE + 2 * TY + 2 * TX;          // tile, left, right, bottom, top
    static constexpr int LX = 4 * N;                            // lines per element and direction
    static constexpr int NBL = (2 * TE + 2 * TY + 2 * TX) * LX; // smoothness lines
    static constexpr size_t bytes = sizeof(double) * (size_t(NSLOT) * ND + size_t(TE) * ND + NBL);
};

// WENOLimiter::compute_smoothness (filter.hpp:586-616) of one line
template <int N> __device__ __forceinline__ double line_smoothness(const StabArgs& a, const double* v)
{
    double cur[N], nxt[N];
#pragma unroll
    for (int i = 0; i < N; ++i) cur[i] = v[i];
    double beta = 0.0, factor = 4.0;
#pragma unroll
    for (int s = 1; s <= N - 1; ++s)
    {
#pragma unroll
        for (int r = 0; r < N; ++r)
        {
            double acc = 0.0;
#pragma unroll
            for (int c = 0; c < N; ++c) acc += a.D[r * N + c] * cur[c];
            nxt[r] = acc;
        }
        double integ = 0.0;
#pragma unroll
        for (int i = 0; i < N; ++i)
        {
            cur[i] = nxt[i];
            integ += a.w[i] * cur[i] * cur[i];
        }
        beta += factor * (0.5 * integ);
        factor *= 4.0;
    }
    return beta;
}

// |x|^theta; theta = 1 (the shock runs' setting) is exactly |x|
__device__ __forceinline__ double sensor_pow(double x, double theta) { return theta == 1.0 ? x : pow(x, theta); }

// One tile (bx, by) of the 2D post-step; stab_smem is the CTA's dynamic shared memory.
template <int N> __device__ __forceinline__ void stab2d_tile(const StabArgs& a, int bx, int by, unsigned char* stab_smem)
{
    using T = StabTile<N>;
    constexpr int TX = T::TX, TY = T::TY, TE = T::TE, ND = T::ND, LX = T::LX;
    double* sU = reinterpret_cast<double*>(stab_smem);
    double* sX = sU + T::NSLOT * ND;
    double* sB = sX + TE * ND;
    const int tid = threadIdx.x;
    const int i0 = bx * TX, j0 = by * TY;
    const int txe = min(TX, a.Nx - i0), tye = min(TY, a.Ny - j0);
    const bool weno = a.apply_weno && !a.apply_filter;
    const int nslot = weno ? T::NSLOT : TE;
    const double igam0 = 1.0 / a.gam[0], igam1 = 1.0 / a.gam[1], igam2 = 1.0 / a.gam[2];

    // global element of a slot, or -1 (outside the tile or a zero ghost across a
    // non-periodic boundary)
    auto slot_elem = [&](int sl) -> int64_t {
        int i, j;
        if (sl < TE)
        {
            const int tx = sl % TX, ty = sl / TX;
            if (tx >= txe || ty >= tye) return -1;
            i = i0 + tx;
            j = j0 + ty;
        }
        else
        {
            const int h = sl - TE;
            if (h < 2 * TY)
            {
                const int ty = h % TY;
                if (ty >= tye) return -1;
                i = h < TY ? i0 - 1 : i0 + txe;
                j = j0 + ty;
            }
            else
            {
                const int tx = (h - 2 * TY) % TX;
                if (tx >= txe) return -1;
                i = i0 + tx;
                j = h < 2 * TY + TX ? j0 - 1 : j0 + tye;
            }
            if (i < 0 || i >= a.Nx)
            {
                if (!a.per_x) return -1;
                i = (i + a.Nx) % a.Nx;
            }
            if (j < 0 || j >= a.Ny)
            {
                if (!a.per_y) return -1;
                j = (j + a.Ny) % a.Ny;
            }
        }
        return int64_t(j) * a.Nx + i;
    };

    // stage the slots (whole elements, 16-byte copies)
    for (int q = tid; q < nslot * (ND / 2); q += kThreads)
    {
        const int sl = q / (ND / 2), k = q % (ND / 2);
        const int64_t ge = slot_elem(sl);
        const double2 v = ge >= 0 ? __ldg(reinterpret_cast<const double2*>(a.src + ge * ND) + k) : make_double2(0.0, 0.0);
        reinterpret_cast<double2*>(sU + sl * ND)[k] = v;
    }
    __syncthreads();

    // values of line li (eq = li % 4, m = li / 4) of a slot in direction dir
    auto line_vals = [&](int sl, int dir, int li, double* v) {
        const int eq = li % 4, m = li / 4;
        const double* base = sU + sl * ND + eq;
#pragma unroll
        for (int t = 0; t < N; ++t) v[t] = base[(dir == 0 ? m * N + t : t * N + m) * 4];
    };

    if (weno)
    {
        // smoothness of every line: tile x-lines, tile y-lines, then the halo slots
        // (left, right: x-lines; bottom, top: y-lines), LX lines each
        for (int b = tid; b < T::NBL; b += kThreads)
        {
            const int blk = b / LX, li = b % LX;
            int sl, dir;
            if (blk < TE) sl = blk, dir = 0;
            else if (blk < 2 * TE) sl = blk - TE, dir = 1;
            else sl = TE + (blk - 2 * TE), dir = (blk - 2 * TE) < 2 * TY ? 0 : 1;
            double v[N];
            line_vals(sl, dir, li, v);
            sB[b] = line_smoothness<N>(a, v);
        }
        __syncthreads();
    }

    // limit the tile lines: x-lines into sX, then y-lines combined with them
#pragma unroll 1
    for (int dir = 0; dir < 2; ++dir)
    {
        for (int q = tid; q < TE * LX; q += kThreads)
        {
            const int e = q / LX, li = q % LX, tx = e % TX, ty = e / TX;
            if (tx >= txe || ty >= tye) continue;
            double cv[N], o[N];
            line_vals(e, dir, li, cv);
            if (weno)
            {
                int sp, sn, bp, bn;
                if (dir == 0)
                {
                    sp = tx > 0 ? e - 1 : TE + ty;
                    bp = tx > 0 ? (e - 1) * LX : (2 * TE + ty) * LX;
                    sn = tx < txe - 1 ? e + 1 : TE + TY + ty;
                    bn = tx < txe - 1 ? (e + 1) * LX : (2 * TE + TY + ty) * LX;
                }
                else
                {
                    sp = ty > 0 ? e - TX : TE + 2 * TY + tx;
                    bp = ty > 0 ? (TE + e - TX) * LX : (2 * TE + 2 * TY + tx) * LX;
                    sn = ty < tye - 1 ? e + TX : TE + 2 * TY + TX + tx;
                    bn = ty < tye - 1 ? (TE + e + TX) * LX : (2 * TE + 2 * TY + TX + tx) * LX;
                }
                const double b0 = sB[bp + li], b1 = sB[(dir * TE + e) * LX + li], b2 = sB[bn + li];
                // ShockSensor::detect_shock (filter.hpp:654-678)
                // divisions as reciprocals and products (within a few ulps of the
                // reference's quotients; the 1/gamma_k are shared by every line)
                // (the reciprocals' range checks deferred: one branch per group instead of
                // one per reciprocal, redone with the checked ones when an input left the
                // fast range; the same results)
                const double x0 = (1.0e-6 + b0) * (1.0e-6 + b0), x1 = (1.0e-6 + b1) * (1.0e-6 + b1),
                             x2 = (1.0e-6 + b2) * (1.0e-6 + b2);
                unsigned bad = 0;
                const MathDeferred md{bad};
                double q0 = md.rcp(x0), q1 = md.rcp(x1), q2 = md.rcp(x2);
                if (bad)
                {
                    q0 = s_rcp(x0);
                    q1 = s_rcp(x1);
                    q2 = s_rcp(x2);
                }
                double cg0 = a.gam[0] * q0;
                double cg1 = a.gam[1] * q1;
                double cg2 = a.gam[2] * q2;
                const double sw = cg0 + cg1 + cg2;
                unsigned bad_w = 0;
                double iws = MathDeferred{bad_w}.rcp(sw);
                if (bad_w) iws = s_rcp(sw);
                cg0 *= iws;
                cg1 *= iws;
                cg2 *= iws;
                const double num = sensor_pow(fabs(cg0 * igam0 - 1.0), a.theta) +
                                   sensor_pow(fabs(cg1 * igam1 - 1.0), a.theta) +
                                   sensor_pow(fabs(cg2 * igam2 - 1.0), a.theta);
                const double r_j = num * a.one_over_norm;
                if (fabs(r_j) >= a.threshold)
                {
                    // WENOLimiter::apply_weno_scalar (filter.hpp:519-544)
                    double pv[N], nv[N];
                    line_vals(sp, dir, li, pv);
                    line_vals(sn, dir, li, nv);
                    double ap = 0.0, ac = 0.0, an = 0.0;
#pragma unroll
                    for (int i = 0; i < N; ++i)
                    {
                        ap += a.w[i] * pv[i];
                        ac += a.w[i] * cv[i];
                        an += a.w[i] * nv[i];
                    }
                    ap *= 0.5;
                    ac *= 0.5;
                    an *= 0.5;
#pragma unroll
                    for (int i = 0; i < N; ++i) o[i] = cg0 * (pv[i] - ap + ac) + cg1 * cv[i] + cg2 * (nv[i] - an + ac);
                }
                else
                {
#pragma unroll
                    for (int i = 0; i < N; ++i) o[i] = cv[i];
                }
            }
            else
            {
                // SpectralFilter::apply_filter (filter.hpp:425-445)
#pragma unroll
                for (int r = 0; r < N; ++r)
                {
                    double acc = 0.0;
#pragma unroll
                    for (int c = 0; c < N; ++c) acc += a.F[r * N + c] * cv[c];
                    o[r] = acc;
                }
            }
            const int eq = li % 4, m = li / 4;
            double* dst = sX + e * ND + eq;
#pragma unroll
            for (int t = 0; t < N; ++t)
            {
                const int node = dir == 0 ? m * N + t : t * N + m;
                dst[node * 4] = dir == 0 ? o[t] : 0.5 * (dst[node * 4] + o[t]);
            }
        }
        __syncthreads();
    }

    // store the tile
    for (int q = tid; q < TE * (ND / 2); q += kThreads)
    {
        const int e = q / (ND / 2), k = q % (ND / 2), tx = e % TX, ty = e / TX;
        if (tx >= txe || ty >= tye) continue;
        reinterpret_cast<double2*>(a.dst + (int64_t(j0 + ty) * a.Nx + (i0 + tx)) * ND)[k] =
            reinterpret_cast<const double2*>(sX + e * ND)[k];
    }
}

// three CTAs per SM at n <= 6 (shared memory allows three there)
template <int N> __global__ void __launch_bounds__(kThreads, N <= 6 ? 3 : 1) stab2d_tile_kernel(const StabArgs a)
{
    extern __shared__ __align__(16) unsigned char stab_smem[];
    stab2d_tile<N>(a, blockIdx.x, blockIdx.y, stab_smem);
}

// The post-step of a batch group: tile t of the list is (instance in group, bx, by);
// the instance's arguments come from device memory into shared memory, inactive
// instances (clock) are skipped.
template <int N> __global__ void __launch_bounds__(kThreads, N <= 6 ? 3 : 1) stab2d_batch_kernel(const StabBatchArgs b)
{
    extern __shared__ __align__(16) unsigned char stab_smem[];
    __shared__ __align__(16) StabArgs sa;
    const int4 tm = b.tiles[blockIdx.x];
    if (!b.clock[b.inst_clock[tm.x]].active) return;
    {
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(b.inst + tm.x);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sa);
        for (int q = threadIdx.x; q < int(sizeof(StabArgs) / 8); q += blockDim.x) dst[q] = src[q];
    }
    __syncthreads();
    stab2d_tile<N>(sa, tm.y, tm.z, stab_smem);
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

// prim_to_cons_elem (problem_def.hpp:36-51) on every node.
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
        using T = StabTile<N>;
        auto kern = stab2d_tile_kernel<N>;
        // the shared-memory opt-in is per device: set it once on each device that launches
        static bool attr_done[64] = {};
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= 64 || !attr_done[dev])
        {
            e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(T::bytes));
            if (e != cudaSuccess) return e;
            if (dev >= 0 && dev < 64) attr_done[dev] = true;
        }
        dim3 grid((a.Nx + T::TX - 1) / T::TX, (a.Ny + T::TY - 1) / T::TY);
        kern<<<grid, kThreads, T::bytes, s>>>(a);
    }
    else
    {
        const int64_t lines = int64_t(a.Nx) * 3;
        stab1d_kernel<N><<<unsigned((lines + kThreads - 1) / kThreads), kThreads, 0, s>>>(a);
    }
    return cudaGetLastError();
}

template <int N> cudaError_t launch_stab_batch_n(const StabBatchArgs& b, cudaStream_t s)
{
    using T = StabTile<N>;
    auto kern = stab2d_batch_kernel<N>;
    static bool attr_done[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64 || !attr_done[dev])
    {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(T::bytes));
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) attr_done[dev] = true;
    }
    if (b.ntiles > 0) kern<<<b.ntiles, kThreads, T::bytes, s>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_stab_batch(int n, const StabBatchArgs& b, cudaStream_t s)
{
    switch (n)
    {
        case 2: return launch_stab_batch_n<2>(b, s);
        case 3: return launch_stab_batch_n<3>(b, s);
        case 4: return launch_stab_batch_n<4>(b, s);
        case 5: return launch_stab_batch_n<5>(b, s);
        case 6: return launch_stab_batch_n<6>(b, s);
        case 7: return launch_stab_batch_n<7>(b, s);
        case 8: return launch_stab_batch_n<8>(b, s);
        case 9: return launch_stab_batch_n<9>(b, s);
        case 10: return launch_stab_batch_n<10>(b, s);
        default: return cudaErrorInvalidValue;
    }
}

void stab_tile_dims(int n, int* tx, int* ty)
{
    const int t = n <= 6 ? 4 : 2;
    *tx = t;
    *ty = t;
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
