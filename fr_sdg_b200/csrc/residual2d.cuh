// residual2d.cuh -- fused FR residual of the 2D Euler equations.
//
// One CTA owns a tile of TX x TY elements and makes one pass over HBM:
//   P1  every tile node: load (with the complex-step seed u + i h v or the
//       prim->cons map applied on the fly), primitives, Euler fluxes F and G to
//       shared memory; element-boundary nodes and the four halo traces also
//       leave a face record (rho, rho u, rho v, rho E, u, v, p, c);
//   P2  one Riemann solve per face point of the tile (faces inside the tile and
//       on its edges, boundary ghosts on physical edges) giving the jumps
//       scale*(F* - F.n) of each adjacent element, and, alongside, the
//       eta-derivatives of each element column;
//   P3  per element row: the xi-derivatives, the chain-rule combination, the four
//       VCJH lifts and the requested output form, stored once.
// Reference: PhysicsEvaluator<Traits,2>::residual_kernel and compute_volume_term,
// include/physics_impl_2D.hpp:268-357 and 646-902, summed in the same order
// (volume, left x-face, right x-face, bottom y-face, top y-face).
// The derivative matrix is read from the kernel-parameter constant bank with
// compile-time indices; tile loops have compile-time trip counts.
#pragma once
#include <cstddef>
#include <type_traits>

#include "device_math.cuh"
#include "frsdg_internal.hpp"
#include "physics.cuh"
#include "pplimit.cuh"
#include "tc_sm100.cuh"

namespace frsdg
{

__host__ __device__ constexpr int round_up32(int v) { return (v + 31) / 32 * 32; }

// Block size and register cap of the 2D kernel (FRSDG_BT / FRSDG_MAXREG override
// them for tuning builds).  A CTA's warps are spread over the SM's four
// sub-partitions, each with a quarter of the register file.
//   face tiles (FP64 at n >= 5, FP32 at n = 5 and 6): one thread per face point of the
//     tile (x-face and y-face threads rounded to warps) plus one warp of element
//     columns (two at n = 5), 80 registers, so that 4-6 CTAs share an SM;
//   otherwise: one thread per tile node (128 to 512), the cap chosen for three
//     co-resident CTAs (one for complex).
// Measured on B200 (1024^2 blast rhs, FP64): p = 4 1.56 -> 1.41 ms, p = 5 1.77 ->
// 1.57 ms, p = 6 4.17 -> 2.91 ms, p = 7 3.48 -> 3.36 ms, p = 8 4.21 -> 3.82 ms,
// p = 9 6.79 -> 4.68 ms; at p = 2 and 3 one thread per node stays ahead (0.52 and
// 0.86 ms against 0.62 and 0.95).  FP32: p = 5 1.00 -> 0.96 ms; at p = 4 one thread
// per node is ahead on the 1024^2 mesh (0.75 against 0.85 ms) but behind on the 64^2
// curved vortex of the mixed-precision runs (0.27 against 0.18 s to t = 10), which
// fills fewer than two waves of CTAs, so FP32 takes face tiles at p = 4 and 5.
__host__ __device__ constexpr int face_threads(int n, int tx, int ty)
{
    return round_up32((tx + 1) * ty * n) + round_up32(tx * (ty + 1) * n);
}
__host__ __device__ constexpr int block_threads(int n, int words, bool f32, int tx, int ty)
{
#ifdef FRSDG_BT
    return FRSDG_BT;
#else
    if (face_tiles(n, words, f32)) return face_threads(n, tx, ty) + (n == 5 ? 64 : 32);
    const int tile_nodes = tx * ty * n * n;
    return round_up32(tile_nodes > 128 ? (tile_nodes < 512 ? tile_nodes : 512) : 128);
#endif
}
__host__ __device__ constexpr int reg_cap(int n, int words, bool f32, int bt)
{
#ifdef FRSDG_MAXREG
    return FRSDG_MAXREG;
#else
    // FP32 at n = 6: 56 registers, six CTAs per SM despite some spills (1024^2 blast
    // 0.89 -> 0.84 ms); at n = 5 the same cap is faster on the 1024^2 mesh (0.79 -> 0.69
    // ms) but slower on the 64^2 curved vortex of the mixed-precision runs (0.18 -> 0.24 s
    // to t = 10), so n = 5 keeps 80.  FP64: 80 registers, no spills.
#ifndef FRSDG_F32_REG6
#define FRSDG_F32_REG6 56
#endif
    if (face_tiles(n, words, f32)) return f32 && n == 6 ? FRSDG_F32_REG6 : 80;
    // three co-resident CTAs (one for complex): per sub-partition ceil(ctas*warps/4) warps
    return (16384 / (32 * (((words == 2 ? 1 : 3) * (bt / 32) + 3) / 4))) / 8 * 8;
#endif
}

// VAR selects the tile: 0 the tuned shape of tile_x/tile_y, 1 the same tile with half
// the element rows (fewer elements per CTA; a candidate of the batch autotuner).
// TC: the FP32 face tiles (n = 5, 6) with the derivative contractions on the tensor
// cores (tc_sm100.cuh); their operands and barrier take a region at the front of the
// shared memory, the tile's usual layout follows it.
template <class S, int N, int GEO, int VAR = 0, bool TC = false> struct Tile2D
{
    static constexpr int W  = scalar_traits<S>::words;
    static constexpr bool F32 = sizeof(S) == 4;
    static constexpr int TX = tile_x(N, W, F32);
    static constexpr int TY = VAR == 0 || tile_y(N, W, F32) == 1 ? tile_y(N, W, F32) : tile_y(N, W, F32) / 2;
    static constexpr int NN = N * N;
    static constexpr int TE = TX * TY;
    static constexpr bool JVP = scalar_traits<S>::words == 2;
    static constexpr int BT = block_threads(N, W, F32, TX, TY);
    // tensor-core tiles: shared memory admits four or five CTAs per SM, so 80 registers
#ifdef FRSDG_TC_MAXREG
    static constexpr int MAXREG = TC ? FRSDG_TC_MAXREG : reg_cap(N, W, F32, BT) > 255 ? 255 : reg_cap(N, W, F32, BT);
#else
    static constexpr int MAXREG = TC ? 80 : reg_cap(N, W, F32, BT) > 255 ? 255 : reg_cap(N, W, F32, BT);
#endif
    static constexpr int NB = 4 * N - 4;  // boundary nodes per element
    static constexpr int NREC_E = TE * NB;
    static constexpr int NHALO  = 2 * TY * N + 2 * TX * N;
    static constexpr int NREC   = NREC_E + NHALO;
    static constexpr int HXL = NREC_E, HXR = HXL + TY * N, HYB = HXR + TY * N, HYT = HYB + TX * N;
    // shared-memory offsets in units of S
    static constexpr int oF   = 0;
    static constexpr int oG   = oF + 4 * TE * NN;
    static constexpr int oC   = oG + 4 * TE * NN;
    static constexpr int oRec = oC + 4 * TE * NN;
    static constexpr int oDel = oRec + RF_N * NREC;
    static constexpr int nS   = oDel + TE * 16 * N;
    static constexpr size_t seed_bytes = JVP ? sizeof(double) * 4 * TE * NN : 0;
    static constexpr size_t bytes = size_t(nS) * sizeof(S) + seed_bytes;
    // stage epilogue (Fr2dArgs::post): the tile's stage outputs, [element][node][eq]
    // doubles, go to the face-record region (dead after P2) when it is large enough,
    // else after the rest; the filter writes its result over the flux region (dead
    // after P3)
    static constexpr size_t post_bytes = size_t(TE) * 4 * NN * sizeof(double);
    static constexpr bool POST_IN_REC = size_t(RF_N) * NREC * sizeof(S) >= post_bytes;
    // tensor-core region: [barrier, TMEM base | A_hi | A_lo | B_hi | B_lo].  The
    // contractions run in two passes through one operand buffer: pass 0 the xi-lines
    // (of F; curved meshes also of G), pass 1 the eta-lines (of G; curved also of F),
    // LSP sets of LINES lines per pass, two 128-line MMA tiles per set.  The second tile
    // of a set reads up to 256 - LINES rows past the set's end: into the next set, or
    // past A_lo into B and the tile region, all inside the CTA's shared memory, and only
    // into accumulator rows nobody reads.  The region is padded so that TMEM columns per
    // byte of shared memory stay below 512 per 228 KB: every mix of these CTAs that fits
    // an SM's shared memory finds its columns free.
    static constexpr int LSP = GEO == GEO_CURVED ? 2 : 1;
    static constexpr int LINES = TE * 4 * N;
    static constexpr int LP = (LINES + 7) / 8 * 8;
    static constexpr int TC_COLS = 2 * LSP * 2 * tc::kCols;  // TMEM columns (a power of two)
    static constexpr size_t tc_a_bytes = size_t(LSP) * LP * tc::kRowBytes;
    static constexpr size_t tc_raw = 128 + 2 * tc_a_bytes + 2 * tc::kBBytes;
    static constexpr size_t tc_min = size_t(TC_COLS) * (228 * 1024 / 512) - 1024 - bytes;
    static constexpr size_t tc_bytes = !TC ? 0 : (tc_raw >= tc_min || tc_min > 1u << 30 ? tc_raw : (tc_min + 127) / 128 * 128);
    static constexpr size_t bytes_post = tc_bytes + (POST_IN_REC ? bytes : bytes + post_bytes);
    static constexpr size_t bytes_launch = tc_bytes + bytes;
    // index of boundary node (k, l) among an element's NB boundary nodes:
    // bottom row, top row, then the interior of the left and right columns
    __host__ __device__ static constexpr int bidx(int k, int l)
    {
        return l == 0 ? k : l == N - 1 ? N + k : k == 0 ? 2 * N + l - 1 : 3 * N - 2 + l - 1;
    }
};

// Load one node's 4 values from the input vectors and form the scalar the residual
// works on: the state itself, M(prim) for the change of variables, or the
// complex-step point M(u + i h v) (petsc_solver_impl.hpp:288-328).
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
            // prim_to_cons_elem (problem_def.hpp:36-51)
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
        const float4 x = __ldg(reinterpret_cast<const float4*>(reinterpret_cast<const float*>(a.U) + off));
        s[0] = x.x; s[1] = x.y; s[2] = x.z; s[3] = x.w;
        if (a.cond_sys)
        {
            const float rho  = expf(s[0]);
            const float ssq  = (0.0f + s[1] * s[1]) + s[2] * s[2];
            const float rhoE = rho * (expf(s[3]) + 0.5f * ssq);
            const float u = s[1], v = s[2];
            s[0] = rho; s[1] = rho * u; s[2] = rho * v; s[3] = rhoE;
        }
    }
};

template <> struct NodeLoader<cplx>
{
    __device__ static void load(const Fr2dArgs& a, int64_t off, cplx s[4])
    {
        const double2 x0 = __ldg(reinterpret_cast<const double2*>(a.U + off));
        const double2 x1 = __ldg(reinterpret_cast<const double2*>(a.U + off + 2));
        double2 v0, v1;
        if (a.mode == MODE_JAC)
        {
            // seed of this launch slice: DOF d of every element of colour c
            const int64_t eg = off / a.nd;
            const int d0 = int(off - eg * a.nd);
            const int gi = int(eg % a.Nx), gj = int(eg / a.Nx);
            const int c = int(blockIdx.z) / a.nd, d = int(blockIdx.z) - c * a.nd;
            const bool on = elem_colour(a.jac_cmode, a.Nx, a.Ny, a.per_x, a.per_y, gi, gj) == c;
            v0 = make_double2(on && d == d0 ? 1.0 : 0.0, on && d == d0 + 1 ? 1.0 : 0.0);
            v1 = make_double2(on && d == d0 + 2 ? 1.0 : 0.0, on && d == d0 + 3 ? 1.0 : 0.0);
        }
        else
        {
            v0 = __ldg(reinterpret_cast<const double2*>(a.W + off));
            v1 = __ldg(reinterpret_cast<const double2*>(a.W + off + 2));
        }
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

template <int GAS, class S>
__device__ __forceinline__ void make_record(const GasParams& g, const S s[4], const NodePrim<S>& pr, S rec[RF_N])
{
    rec[RF_RHO] = s[0];
    rec[RF_E]   = s[3];
    rec[RF_U]   = pr.u;
    rec[RF_V]   = pr.v;
    rec[RF_P]   = pr.p;
    rec[RF_C]   = node_sound_speed<GAS>(g, pr);
}

template <class S> struct Rec
{
    S v[RF_N];
};

// The FP32 instantiation reading an FP64 state (a.in_f64, the mixed form): the node's
// state is loaded in FP64 and its primitives (density, velocities, internal energy,
// pressure, and the sound speed when asked) are recovered in FP64 before rounding to
// FP32, so that pressures near vacuum keep their sign; fluxes, Riemann solves and
// derivatives then run in FP32.  Returns whether it took that path.
template <int GAS, class S, class M = MathChecked>
__device__ __forceinline__ bool node_state_f64(const Fr2dArgs& a, const GasParams& g, int64_t off, S s[4],
                                               NodePrim<S>& pr, S* c, const M& m = M{})
{
    if constexpr (sizeof(S) == 4)
    {
        if (a.in_f64)
        {
            double d[4];
            NodeLoader<double>::load(a, off, d);
            const NodePrim<double> q = node_prim<GAS>(g, d[0], d[1], d[2], d[3], m);
#pragma unroll
            for (int i = 0; i < 4; ++i) s[i] = static_cast<float>(d[i]);
            pr.rho_w = static_cast<float>(q.rho_w);
            pr.inv_rho = static_cast<float>(q.inv_rho);
            pr.u = static_cast<float>(q.u);
            pr.v = static_cast<float>(q.v);
            pr.e = static_cast<float>(q.e);
            pr.p = static_cast<float>(q.p);
            pr.inv_covol = static_cast<float>(q.inv_covol);
            if (c) *c = static_cast<float>(node_sound_speed<GAS>(g, q, m));
            return true;
        }
    }
    return false;
}

// Boundary ghost record on a physical edge from the interior node's state (rare
// path, kept out of line; the record returns by value).
template <int GAS, class S>
__device__ __noinline__ Rec<S> ghost_record(const Fr2dArgs& a, int dir, int64_t interior_off, double x, double y,
                                            double nx, double ny)
{
    Rec<S> out;
    if constexpr (sizeof(S) == 4)
    {
        if (a.in_f64)
        {
            double d_in[4], d_out[4];
            NodeLoader<double>::load(a, interior_off, d_in);
            bc_ghost2<GAS>(a.bc[dir], dir, a.gas, a.t, x, y, nx, ny, a.Lx, a.Ly, d_in, d_out, false);
            const NodePrim<double> q = node_prim<GAS>(a.gas, d_out[0], d_out[1], d_out[2], d_out[3]);
            double r[RF_N];
            make_record<GAS>(a.gas, d_out, q, r);
#pragma unroll
            for (int f = 0; f < RF_N; ++f) out.v[f] = static_cast<float>(r[f]);
            return out;
        }
    }
    S s_in[4], s_out[4];
    NodeLoader<S>::load(a, interior_off, s_in);
    bc_ghost2<GAS>(a.bc[dir], dir, a.gas, a.t, x, y, nx, ny, a.Lx, a.Ly, s_in, s_out, a.exact_bc != 0);
    const NodePrim<S> pr = node_prim<GAS>(a.gas, s_out[0], s_out[1], s_out[2], s_out[3]);
    make_record<GAS>(a.gas, s_out, pr, out.v);
    return out;
}

// One side of a face point: its record, whether it is a tile element (and which
// element/node) or a physical-boundary ghost, and the face normal.
template <class S> struct FaceSide
{
    S R[RF_N];
    double nx, ny;
    int e, node;     // tile element and node of this side (e < 0: halo or ghost)
    bool bc;         // ghost from a boundary condition
};

// Locate face point t of the x-faces (XF) or y-faces of the tile, fetch both
// side records.  Returns false (with harmless records) when t is not a face point.
template <class S, int N, int GEO, bool XF, class T>
__device__ __forceinline__ bool face_prepare(const Fr2dArgs& a, bool exists, int t, int i0, int j0, int txe,
                                             int tye, const S* sRec, FaceSide<S> sd[2])
{
    constexpr int TX = T::TX, NREC = T::NREC;
    const int pos = t % N, r = t / N;
    int face, row, lim;
    if constexpr (XF)
    {
        face = r % (TX + 1);
        row = r / (TX + 1);
        lim = txe;
        exists = exists && row < tye && face <= txe;
    }
    else
    {
        row = r % TX;
        face = r / TX;
        lim = tye;
        exists = exists && face <= tye && row < txe;
    }
    const int gI = XF ? i0 + face : i0 + row;
    const int gJ = XF ? j0 + row : j0 + face;
    double nx = XF ? 1.0 : 0.0, ny = XF ? 0.0 : 1.0;
    if constexpr (GEO == GEO_CURVED)
    {
        if (exists)
        {
            const double2 nn = XF ? __ldg(reinterpret_cast<const double2*>(a.xnorm) + (int64_t(gJ + a.row_base) * (a.Nx + 1) + gI) * N + pos)
                                  : __ldg(reinterpret_cast<const double2*>(a.ynorm) + (int64_t(gJ + a.row_base) * a.Nx + gI) * N + pos);
            nx = nn.x;
            ny = nn.y;
        }
    }
    const bool inM = exists && face > 0, inP = exists && face < lim;
    const bool per = XF ? a.per_x : a.per_y;
    const int  gface = XF ? gI : gJ, gmax = XF ? a.Nx : a.Ny;
    const bool bcM = exists && face == 0 && gface == 0 && !per;
    const bool bcP = exists && face == lim && gface == gmax && !per;
    const int eM = XF ? row * TX + face - 1 : (face - 1) * TX + row;
    const int eP = XF ? row * TX + face : face * TX + row;
    const int nodeM = XF ? pos * N + (N - 1) : (N - 1) * N + pos;
    const int nodeP = XF ? pos * N : pos;
    int rM = inM ? eM * T::NB + (XF ? T::bidx(N - 1, pos) : T::bidx(pos, N - 1))
                 : (XF ? T::HXL : T::HYB) + row * N + pos;
    int rP = inP ? eP * T::NB + (XF ? T::bidx(0, pos) : T::bidx(pos, 0))
                 : (XF ? T::HXR : T::HYT) + row * N + pos;
    if (!exists || bcM) rM = 0;  // any valid record keeps the arithmetic finite
    if (!exists || bcP) rP = 0;
#pragma unroll
    for (int f = 0; f < RF_N; ++f)
    {
        sd[0].R[f] = sRec[f * NREC + rM];
        sd[1].R[f] = sRec[f * NREC + rP];
    }
    sd[0].nx = sd[1].nx = nx;
    sd[0].ny = sd[1].ny = ny;
    sd[0].e = inM ? eM : -1;
    sd[1].e = inP ? eP : -1;
    sd[0].node = nodeM;
    sd[1].node = nodeP;
    sd[0].bc = bcM;
    sd[1].bc = bcP;
    // the ghost needs the global position of the face point and of its interior node
    if (bcM) sd[0].e = -2 - (XF ? (gJ + a.row_base) * N + pos : gI * N + pos), sd[1].e = eP;
    if (bcP) sd[1].e = -2 - (XF ? (gJ + a.row_base) * N + pos : gI * N + pos), sd[0].e = eM;
    return exists;
}

// Replace the record of a boundary side by its ghost (rare path).
template <int GAS, class S, int N, bool XF, class T>
__device__ __forceinline__ void face_ghost(const Fr2dArgs& a, int i0, int j0, FaceSide<S> sd[2])
{
    constexpr int TX = T::TX, NN = N * N;
#pragma unroll
    for (int side = 0; side < 2; ++side)
    {
        if (!sd[side].bc) continue;
        const int dir = XF ? (side == 0 ? FRSDG_LEFT : FRSDG_RIGHT) : (side == 0 ? FRSDG_BOTTOM : FRSDG_TOP);
        const int bi = -2 - sd[side].e;
        const double2 xy = __ldg(reinterpret_cast<const double2*>(a.bxy[dir]) + bi);
        const FaceSide<S>& in = sd[1 - side];
        const int64_t ioff = (int64_t(j0 + in.e / TX) * a.Nx + (i0 + in.e % TX)) * (4 * NN) + in.node * 4;
        const Rec<S> gh = ghost_record<GAS, S>(a, dir, ioff, xy.x, xy.y, sd[side].nx, sd[side].ny);
#pragma unroll
        for (int f = 0; f < RF_N; ++f) sd[side].R[f] = gh.v[f];
        sd[side].e = -1;
    }
}

// Jumps scale*(F* - F.n) of the tile sides of a face point; F.n from the cached
// volume fluxes (F.n = F on affine x-faces, G on affine y-faces).
template <class S, int N, int GEO, bool XF, class T>
__device__ __forceinline__ void face_jumps(const Fr2dArgs& a, int i0, int j0, bool valid, const FaceSide<S> sd[2],
                                           const S Fs[4], const S* sF, const S* sG, S* sDel)
{
    constexpr int TX = T::TX, NN = N * N;
    using R_t = typename scalar_traits<S>::real;
    if (!valid) return;
#pragma unroll
    for (int side = 0; side < 2; ++side)
    {
        const int e = sd[side].e;
        if (e < 0) continue;
        const int node = sd[side].node;
        double sc;
        if constexpr (GEO == GEO_CURVED)
        {
            const double* mt = a.metrics + ((int64_t(j0 + e / TX + a.row_base) * a.Nx + (i0 + e % TX)) * NN + node) * 4 + (XF ? 0 : 2);
            const double2 m = __ldg(reinterpret_cast<const double2*>(mt));
            sc = sqrt(m.x * m.x + m.y * m.y);
        }
        else
            sc = XF ? a.scale_x : a.scale_y;
        const int sdi = XF ? (side == 0 ? 1 : 0) : (side == 0 ? 3 : 2);
        const int pos = XF ? node / N : node % N;
#pragma unroll
        for (int eq = 0; eq < 4; ++eq)
        {
            S fn;
            if constexpr (GEO == GEO_CURVED)
                fn = sF[(e * 4 + eq) * NN + node] * R_t(sd[side].nx) + sG[(e * 4 + eq) * NN + node] * R_t(sd[side].ny);
            else
                fn = XF ? sF[(e * 4 + eq) * NN + node] : sG[(e * 4 + eq) * NN + node];
            sDel[((e * 4 + sdi) * 4 + eq) * N + pos] = R_t(sc) * (Fs[eq] - fn);
        }
    }
}

// Stage epilogue of a tile (Fr2dArgs::post, MODE_STAGE): sO holds the stage outputs of
// the tile's elements; the spectral filter of the post-step (stab2d_tile's filter
// branch, SpectralFilter::apply_filter, filter.hpp:425-445: half the sum of the filter
// along the element's rows and along its columns), the positivity limiter and the
// wave-speed maximum act on each element in shared memory, then the tile is stored.
template <class T, int N, int GAS>
__device__ __forceinline__ void stage_epilogue(const Fr2dArgs& a, const Ops& ops, int i0, int j0, int txe, int tye,
                                               double* sO, unsigned char* smem_raw)
{
    constexpr int TX = T::TX, TE = T::TE, BT = T::BT, NN = N * N, ND = 4 * NN;
    static_assert(BT % 32 == 0, "whole warps");
    const int tid = threadIdx.x;
    const PostArgs& P = *a.pa;
    const bool filter = (a.post & POST_FILTER) != 0;
    __shared__ int s_flag[TE];  // elements the limiter changed (their stored values are stale)
    for (int e = tid; e < TE; e += BT) s_flag[e] = 0;
    double* sX = sO;
    if (a.post & POST_FILTER)
    {
        double* sY = reinterpret_cast<double*>(smem_raw);
#pragma unroll 1
        for (int dir = 0; dir < 2; ++dir)
        {
            for (int t = tid; t < TE * 4 * N; t += BT)
            {
                const int eq = t % 4, m = (t / 4) % N, e = t / (4 * N);
                if (e % TX >= txe || e / TX >= tye) continue;
                const double* src = sO + e * ND + eq;
                double cv[N];
#pragma unroll
                for (int c = 0; c < N; ++c) cv[c] = src[(dir == 0 ? m * N + c : c * N + m) * 4];
#pragma unroll
                for (int r = 0; r < N; ++r)
                {
                    double acc = 0.0;
#pragma unroll
                    for (int c = 0; c < N; ++c) acc += ops.F[r * N + c] * cv[c];
                    double& d = sY[e * ND + (dir == 0 ? m * N + r : r * N + m) * 4 + eq];
                    d = dir == 0 ? acc : 0.5 * (d + acc);
                }
            }
            __syncthreads();
        }
        sX = sY;
    }
    if (a.post & (POST_PP | POST_AMAX))
    {
        // screen every node of the tile at once (pp_element2d's test: density and
        // pressure above the floor leave the element as it is); only the elements with
        // a node below it go through the limiter, one warp each.  Clear elements give
        // their wave speeds here, limited ones after limiting.
        const PPView v{GAS == 0 ? FRSDG_GAS_IDEAL : FRSDG_GAS_VDW, a.gas, P.pp_eps, P.w, P.detJ};
        const bool limit = (a.post & POST_PP) != 0, want_amax = (a.post & POST_AMAX) != 0;
        __shared__ unsigned long long s_amax;
        if (tid == 0) s_amax = 0ull;
        __syncthreads();
        const double thr = v.eps0 * (1.0 + 1e-10);
        double w = 0.0;
        for (int q = tid; q < TE * NN; q += BT)
        {
            const int e = q / NN;
            if (e % TX >= txe || e / TX >= tye) continue;
            const double2 x0 = *reinterpret_cast<const double2*>(sX + q * 4);
            const double2 x1 = *reinterpret_cast<const double2*>(sX + q * 4 + 2);
            const double u[4] = {x0.x, x0.y, x1.x, x1.y};
            if (limit)
            {
                unsigned bad = 0;
                double p = pp_pressure_fast(v, u, MathDeferred{bad});
                if (bad) p = pp_pressure_fast(v, u);
                if (!(u[0] > thr && p > thr))
                {
                    s_flag[e] = 1;
                    continue;
                }
            }
            if (want_amax) w = fmax(w, node_wave_speed_fast(v, u));
        }
        if (want_amax)
        {
            w = -pp_warp_min(-w);
            if ((tid & 31) == 0 && w > 0.0 && w < 1e300)
                atomicMax(&s_amax, static_cast<unsigned long long>(__double_as_longlong(w)));
        }
        __syncthreads();
        if (limit)
        {
            unsigned long long* amax = want_amax ? &s_amax : nullptr;
            for (int e = tid / 32; e < TE; e += BT / 32)
            {
                const int tx = e % TX, ty = e / TX;
                if (tx >= txe || ty >= tye || !s_flag[e]) continue;  // uniform across the warp
                const int64_t e_glob = int64_t(j0 + ty + a.row_base) * a.Nx + (i0 + tx);
                pp_element2d<N>(v, sX + e * ND, nullptr, e_glob, true, false, amax);
            }
            __syncthreads();
        }
        if (want_amax && tid == 0 && s_amax) atomicMax(P.amax, s_amax);
    }
    // store: the filtered tile, or (values already stored by the row pass) the
    // elements the limiter changed
    if (!filter && !(a.post & POST_PP)) return;
    if (!filter) __syncthreads();  // s_flag complete (the limiter's own barrier may be skipped)
    double* out = static_cast<double*>(a.out);
    for (int q = tid; q < TE * (ND / 2); q += BT)
    {
        const int e = q / (ND / 2), k = q % (ND / 2), tx = e % TX, ty = e / TX;
        if (tx >= txe || ty >= tye || !(filter || s_flag[e])) continue;
        reinterpret_cast<double2*>(out + (int64_t(j0 + ty) * a.Nx + (i0 + tx)) * ND)[k] =
            reinterpret_cast<const double2*>(sX + e * ND)[k];
    }
}

// One tile of the residual pass: tile (bx, by) of element columns/rows (the Jacobian
// slice of MODE_JAC is blockIdx.z), with the launch arguments `a` and the operators
// `ops`; smem_raw is the CTA's dynamic shared memory (T::bytes).
// FP32 derivatives: the rows of the rounded differentiation matrix do not sum to zero
// exactly, so a line's constant part (a uniform background flux) would leave a residual
// of ~1e-7 |F| |D| at every node, the same sign every step.  Differentiating the line
// minus its first value removes that bias (D 1 = 0 in exact arithmetic, so the result
// is unchanged otherwise).  FP64 keeps the reference's form.
template <class S, int N> __device__ __forceinline__ void center_line(S (&v)[N])
{
    if constexpr (sizeof(S) == 4)
    {
        const S b = v[0];
#pragma unroll
        for (int m = 0; m < N; ++m) v[m] = v[m] - b;
    }
}

// POST: the instantiation with the stage epilogue (Fr2dArgs::post); the others carry no
// epilogue code, which would otherwise cost the main path registers.
template <class S, int N, int GAS, int RIEM, int GEO, int VAR, bool POST = false, bool TC = false>
__device__ __forceinline__ void fr2d_tile(const Fr2dArgs& a, const Ops& ops, int bx, int by, unsigned char* smem_raw)
{
    using T = Tile2D<S, N, GEO, VAR, TC>;
    constexpr int TX = T::TX, TY = T::TY, NN = T::NN, TE = T::TE, BT = T::BT, NREC = T::NREC;
    using R_t = typename scalar_traits<S>::real;
    constexpr int ND = 4 * NN;
    static_assert(!TC || (T::F32 && N >= 5 && N <= 8), "tensor-core contractions: FP32 at n = 5..8");
    static_assert(!TC || (T::LINES <= BT && BT <= 2 * tc::kTileLines), "one line of each set per thread");
    // every CTA of every mix of these kernels that fits on an SM (228 KB of shared memory)
    // finds its TMEM columns free: columns per byte of shared memory stay below 512 / 228 KB
    static_assert(!TC || size_t(T::TC_COLS) * (228 * 1024) <= size_t(512) * (T::bytes_launch + 1024),
                  "TMEM columns per CTA against shared memory per CTA");
    unsigned char* base = smem_raw + T::tc_bytes;  // the tile's layout (tensor-core region first)
    S* sm   = reinterpret_cast<S*>(base);
    S* sF   = sm + T::oF;
    S* sG   = sm + T::oG;
    S* sC   = sm + T::oC;
    S* sRec = sm + T::oRec;
    S* sDel = sm + T::oDel;
    // stage epilogue: the tile's stage outputs (Tile2D::POST_IN_REC)
    // (POST instantiations run only stage launches: the launcher and the batch kernel)
    constexpr bool post = POST && !T::JVP;
    double* sO = reinterpret_cast<double*>(base + (T::POST_IN_REC ? T::oRec * sizeof(S) : T::bytes));
    double* sSeed = reinterpret_cast<double*>(base + size_t(T::nS) * sizeof(S));
    // tensor-core region
    uint64_t* tc_bar = reinterpret_cast<uint64_t*>(smem_raw);
    uint32_t* tc_tmem = reinterpret_cast<uint32_t*>(smem_raw + 8);
    unsigned char* tc_ahi = smem_raw + 128;
    unsigned char* tc_alo = tc_ahi + T::tc_a_bytes;
    unsigned char* tc_bhi = tc_alo + T::tc_a_bytes;
    unsigned char* tc_blo = tc_bhi + tc::kBBytes;

    const int tid = threadIdx.x;
    const int Nx = a.Nx, Ny = a.Ny;
    const int i0 = bx * TX, j0 = by * TY + a.row_begin;
    const int txe = min(TX, Nx - i0), tye = min(TY, a.row_end - j0);
    const GasParams g = a.gas;

    if constexpr (TC)
    {
        // TMEM for the accumulators (warp 0), the MMA-completion barrier, and the split
        // differentiation matrix as the B operand (16 rows)
        if (tid < 32) tc::tmem_alloc(tc_tmem, T::TC_COLS);
        else if (tid == 32) tc::mbar_init(tc_bar, 1);
        else if (tid >= 64 && tid < 64 + tc::kCols) tc::pack_matrix_row<N>(tc_bhi, tc_blo, tid - 64, ops.D);
    }

    if constexpr (!T::JVP)
    {
        // Epilogue operands (RK stage: A and B; IFunction: U_t): pull the tile's lines
        // into L2 first, so that their reads after the face phase do not wait on HBM
        // (prefetches are hints; measured: SSP-RK3 stage on the 1024^2 p5 blast 1.95 ->
        // 1.74 ms)
        if (a.mode == MODE_STAGE || a.mode == MODE_IFUNC)
        {
            constexpr int LROW = (TX * ND * int(sizeof(double)) + 127) / 128;  // 128-byte lines per tile row
            const int lrow = (txe * ND * int(sizeof(double)) + 127) / 128;
            const double* b0 = a.mode == MODE_STAGE ? a.st.A : a.W;
            const double* b1 = a.mode == MODE_STAGE ? a.st.B : nullptr;
            for (int q = tid; q < 2 * TY * LROW; q += BT)
            {
                const int which = q / (TY * LROW), r = q % (TY * LROW), ty = r / LROW, ln = r % LROW;
                const double* base = which ? b1 : b0;
                if (base && ty < tye && ln < lrow)
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(base + (int64_t(j0 + ty) * Nx + i0) * ND + ln * 16));
            }
        }
    }

    // ---- P1: nodes of the tile; the halo traces (x-left, x-right per tile row,
    // y-bottom, y-top per tile column) are fetched first so their latency overlaps
    static_assert(T::NHALO <= BT, "one halo node per thread");
    S hs[4];
    int hrec = -1;
    int64_t hoff = 0;
    // the last NHALO threads carry the halo: the first threads may own two tile nodes
    if (tid >= BT - T::NHALO)
    {
        const int q = tid - (BT - T::NHALO);
        int ge_i, ge_j, node, r;
        bool ok;
        if (q < 2 * TY * N)
        {
            const int side = q / (TY * N), ty = (q % (TY * N)) / N, m = q % N;
            ok = ty < tye;
            ge_j = j0 + ty;
            if (side == 0)
            {
                ge_i = i0 - 1;
                if (ge_i < 0) { ok = ok && a.per_x; ge_i += Nx; }
                node = m * N + (N - 1);
                r = T::HXL + ty * N + m;
            }
            else
            {
                ge_i = i0 + txe;
                if (ge_i >= Nx) { ok = ok && a.per_x; ge_i -= Nx; }
                node = m * N;
                r = T::HXR + ty * N + m;
            }
        }
        else
        {
            const int qq = q - 2 * TY * N;
            const int side = qq / (TX * N), tx = (qq % (TX * N)) / N, m = qq % N;
            ok = tx < txe;
            ge_i = i0 + tx;
            if (side == 0)
            {
                ge_j = j0 - 1;
                if (ge_j < 0) { ok = ok && a.per_y; ge_j += Ny; }
                node = (N - 1) * N + m;
                r = T::HYB + tx * N + m;
            }
            else
            {
                ge_j = j0 + tye;
                if (ge_j >= Ny) { ok = ok && a.per_y; ge_j -= Ny; }
                node = m;
                r = T::HYT + tx * N + m;
            }
        }
        if (ok)
        {
            hoff = (int64_t(ge_j) * Nx + ge_i) * ND + node * 4;
            if (!(T::F32 && a.in_f64)) NodeLoader<S>::load(a, hoff, hs);
            hrec = r;
        }
    }
    // One tile node: load, primitives, fluxes to sF / sG and (boundary nodes) the face
    // record.  Run with MathDeferred, `bad` tells whether a reciprocal or square root met
    // an input outside the fast range; such nodes are redone after the loop with
    // MathChecked, so that the loop itself stays free of those branches.  (A halo record
    // must equal, bit for bit, the record of the same node computed inside a tile, since
    // row windows move tile edges: node_prim and node_sound_speed pin their operations
    // with explicit multiply-adds, so that every inlined copy rounds alike.)
    auto node_pass = [&](int q, const auto& m) {
        const int e = q / NN, node = q % NN, tx = e % TX, ty = e / TX, k = node % N, l = node / N;
        if (tx < txe && ty < tye)
        {
            const int64_t off = (int64_t(j0 + ty) * Nx + (i0 + tx)) * ND + node * 4;
            const bool bnode = k == 0 || k == N - 1 || l == 0 || l == N - 1;
            S s[4], c = S(0.0);
            NodePrim<S> pr;
            // the sound speed of every node, although only boundary nodes keep a record: a
            // branch on bnode diverges in nearly every warp (1.4 % of the residual's time)
            const bool f64 = node_state_f64<GAS>(a, g, off, s, pr, &c, m);
            if (!f64) NodeLoader<S>::load(a, off, s);
            if constexpr (T::JVP)
            {
#pragma unroll
                for (int eq = 0; eq < 4; ++eq) sSeed[(e * 4 + eq) * NN + node] = s_im(s[eq]);
            }
            if (!f64)
            {
                pr = node_prim<GAS>(g, s[0], s[1], s[2], s[3], m);
                if constexpr (T::JVP)
                {
                    if (bnode) c = node_sound_speed<GAS>(g, pr, m);  // a complex square root
                }
                else
                    c = node_sound_speed<GAS>(g, pr, m);
            }
            const S rEp = s[3] + pr.p;
            const S ruv = s[1] * pr.v;
            S* f = sF + e * 4 * NN + node;
            S* gg = sG + e * 4 * NN + node;
            f[0 * NN] = s[1];
            f[1 * NN] = s[1] * pr.u + pr.p;
            f[2 * NN] = ruv;
            f[3 * NN] = pr.u * rEp;
            gg[0 * NN] = s[2];
            gg[1 * NN] = ruv;
            gg[2 * NN] = s[2] * pr.v + pr.p;
            gg[3 * NN] = pr.v * rEp;
            if (bnode)
            {
                const S rec[RF_N] = {s[0], s[3], pr.u, pr.v, pr.p, c};
                const int r = e * T::NB + T::bidx(k, l);
#pragma unroll
                for (int fld = 0; fld < RF_N; ++fld) sRec[fld * NREC + r] = rec[fld];
            }
            return s_re(s[0]);
        }
        return 1.0;
    };
    auto halo_pass = [&](const auto& m) {
        NodePrim<S> pr;
        S c = S(0.0);
        const bool f64 = node_state_f64<GAS>(a, g, hoff, hs, pr, &c, m);
        if (!f64)
        {
            pr = node_prim<GAS>(g, hs[0], hs[1], hs[2], hs[3], m);
            c = node_sound_speed<GAS>(g, pr, m);
        }
        const S rec[RF_N] = {hs[0], hs[3], pr.u, pr.v, pr.p, c};
#pragma unroll
        for (int fld = 0; fld < RF_N; ++fld) sRec[fld * NREC + hrec] = rec[fld];
    };
    static_assert((TE * NN + BT - 1) / BT < 31, "node iterations fit the redo mask");
    unsigned redo = 0;  // bit i: this thread's node i (bit 31: its halo node) to redo
    {
        int it = 0;
        for (int q = tid; q < TE * NN; q += BT, ++it)
        {
            unsigned bad = 0;
            const double rho = node_pass(q, MathDeferred{bad});
            if (!density_ok(rho) && a.bad) atomicAdd(a.bad, 1ull);
            redo |= bad << it;
        }
        if (hrec >= 0)
        {
            unsigned bad = 0;
            halo_pass(MathDeferred{bad});
            redo |= bad << 31;
        }
    }
    if (redo)
    {
        int it = 0;
        for (int q = tid; q < TE * NN; q += BT, ++it)
            if ((redo >> it) & 1u) node_pass(q, MathChecked{});
        if (redo >> 31) halo_pass(MathChecked{});
    }
    if constexpr (TC)
    {
        tc::fence_async_smem();
        tc::fence_before_sync();
    }
    __syncthreads();
    uint32_t tmem = 0;
    // tensor cores: the flux lines of one pass, each minus its first value (center_line),
    // split into TF32 high and low parts as the A operands of the shared buffer, by the
    // threads first, first + stride, ...; and the MMAs of a pass, issued by one thread
    auto tc_pack = [&](int pass, int first, int stride) {
        if constexpr (TC)
        {
            for (int q = first; q < T::LSP * T::LINES; q += stride)
            {
                const int set = q / T::LINES, t = q % T::LINES;
                const int eq = t % 4, l = (t / 4) % N, e = t / (4 * N);
                const bool xi = pass == 0;
                const S* src = ((set == 0) == xi ? sF : sG) + (e * 4 + eq) * NN + (xi ? l * N : l);
                S v[N];
#pragma unroll
                for (int m = 0; m < N; ++m) v[m] = src[xi ? m : m * N];
                center_line<S, N>(v);
                tc::pack_line<N>(tc_ahi, tc_alo, set * T::LP + t, v);
            }
        }
    };
    auto tc_issue = [&](int pass) {
        if constexpr (TC)
        {
            const uint32_t ah = tc::smem_u32(tc_ahi), al = tc::smem_u32(tc_alo);
            const uint32_t bh = tc::smem_u32(tc_bhi), bl = tc::smem_u32(tc_blo);
#pragma unroll
            for (int set = 0; set < T::LSP; ++set)
            {
#pragma unroll
                for (int q = 0; q < 2; ++q)
                {
                    const uint32_t off = uint32_t(set * T::LP + q * tc::kTileLines) * tc::kRowBytes;
                    tc::split_product(tmem, uint32_t((pass * T::LSP + set) * 2 + q) * tc::kCols, ah + off, al + off,
                                      bh, bl);
                }
            }
            tc::mma_commit(tc_bar);
        }
    };
    if constexpr (TC)
    {
        // pass 0 (xi-lines) by every thread; its MMAs run while the face phase solves its
        // Riemann problems, and the column warps pack and issue pass 1 once they are done
        tc::fence_after_sync();
        tmem = *tc_tmem;
        tc_pack(0, tid, BT);
        tc::fence_async_smem();
        __syncthreads();
        if (tid == 0) tc_issue(0);
    }

    // ---- P2: face points and element columns.  When the block has threads to
    // spare, each face thread solves one face point (x-faces, then y-faces, on
    // separate warps) and the remaining warps differentiate the element columns;
    // otherwise each face thread solves one x-face and one y-face point (two
    // independent Riemann problems in flight) and the columns follow.
    constexpr int NXF = (TX + 1) * TY * N, NYF = TX * (TY + 1) * N, NCOL = TE * 4 * N;
    constexpr int NFP = NXF > NYF ? NXF : NYF;
    constexpr int PFP = round_up32(NFP), PCOL = round_up32(NCOL);
    constexpr int PX = round_up32(NXF), PY = round_up32(NYF);
#ifdef FRSDG_PAIRED
    constexpr bool UNPAIR = false;
#else
    constexpr bool UNPAIR = PX + PY < BT;
#endif
    auto column = [&](int tt) {
        // column (e, eq, k): eta-derivatives of G (and of F on curved meshes)
        const int k = tt % N, r = tt / N, eq = r % 4, e = r / 4;
        if ((e % TX) >= txe || (e / TX) >= tye) return;
        const S* Gc = sG + (e * 4 + eq) * NN + k;
        S gv[N];
#pragma unroll
        for (int m = 0; m < N; ++m) gv[m] = Gc[m * N];
        center_line<S, N>(gv);
        if constexpr (GEO == GEO_CURVED)
        {
            const S* Fc = sF + (e * 4 + eq) * NN + k;
            S fv[N];
#pragma unroll
            for (int m = 0; m < N; ++m) fv[m] = Fc[m * N];
            center_line<S, N>(fv);
            const double* mt = a.metrics + ((int64_t(j0 + e / TX + a.row_base) * Nx + (i0 + e % TX)) * NN + k) * 4 + 2;
#pragma unroll
            for (int l = 0; l < N; ++l)
            {
                S dG = S(0.0), dF = S(0.0);
#pragma unroll
                for (int m = 0; m < N; ++m)
                {
                    dG = dG + opD<R_t>(ops, l * N + m) * gv[m];
                    dF = dF + opD<R_t>(ops, l * N + m) * fv[m];
                }
                const double2 me = __ldg(reinterpret_cast<const double2*>(mt + l * N * 4));
                sC[(e * 4 + eq) * NN + l * N + k] = R_t(me.x) * dF + R_t(me.y) * dG;
            }
        }
        else
        {
#pragma unroll
            for (int l = 0; l < N; ++l)
            {
                S dG = S(0.0);
#pragma unroll
                for (int m = 0; m < N; ++m) dG = dG + opD<R_t>(ops, l * N + m) * gv[m];
                sC[(e * 4 + eq) * NN + l * N + k] = R_t(a.eta_y) * dG;
            }
        }
    };
    // One face point (x-faces: XF): both side records, the boundary ghost, the Riemann
    // flux and the jumps; with MathDeferred, `bad` tells whether to redo it with
    // MathChecked (after the hot code, like the node pass).
    auto face_point = [&](auto xf_tag, int t, bool exists, const auto& m) {
        constexpr bool XF = decltype(xf_tag)::value;
        FaceSide<S> sd[2];
        S Fs[4];
        if (face_prepare<S, N, GEO, XF, T>(a, exists, t, i0, j0, txe, tye, sRec, sd))
        {
            if (sd[0].bc || sd[1].bc) face_ghost<GAS, S, N, XF, T>(a, i0, j0, sd);
            riemann_rec<RIEM>(sd[0].R, sd[1].R, sd[0].nx, sd[0].ny, Fs, m);
            face_jumps<S, N, GEO, XF, T>(a, i0, j0, true, sd, Fs, sF, sG, sDel);
        }
    };
    using XFace = std::true_type;
    using YFace = std::false_type;
    if constexpr (UNPAIR)
    {
        if (tid < PX + PY)
        {
            const bool xf = tid < PX;
            const int t = xf ? tid : tid - PX;
            unsigned bad = 0;
            if (xf)
                face_point(XFace{}, t, t < NXF, MathDeferred{bad});
            else
                face_point(YFace{}, t, t < NYF, MathDeferred{bad});
            if (bad)
            {
                if (xf)
                    face_point(XFace{}, t, t < NXF, MathChecked{});
                else
                    face_point(YFace{}, t, t < NYF, MathChecked{});
            }
        }
        else if constexpr (!TC)
        {
            for (int c = tid - PX - PY; c < NCOL; c += BT - PX - PY) column(c);
        }
        else
        {
            // the column warps: once pass 0's MMAs have read the buffer (barrier phase 0),
            // pack pass 1 (eta-lines) into it and issue its MMAs (phase 1)
            constexpr int NCW = BT - PX - PY;
            static_assert(NCW % 32 == 0 && NCW > 0, "whole column warps");
            if (!tc::mbar_wait(tc_bar, 0, 1 << 20) && a.bad) atomicAdd(a.bad, 1ull << 32);
            tc_pack(1, tid - PX - PY, NCW);
            tc::fence_async_smem();
            if constexpr (NCW == 32)
                __syncwarp();
            else
                asm volatile("bar.sync 1, %0;" ::"n"(NCW) : "memory");
            if (tid == PX + PY) tc_issue(1);
        }
    }
    else
    {
        for (int t = tid; t < PFP + PCOL; t += BT)
        {
            if (t < PFP)
            {
                FaceSide<S> xs[2], ys[2];
                const bool vx = face_prepare<S, N, GEO, true, T>(a, t < NXF, t, i0, j0, txe, tye, sRec, xs);
                const bool vy = face_prepare<S, N, GEO, false, T>(a, t < NYF, t, i0, j0, txe, tye, sRec, ys);
                if (!vx && !vy) continue;
                if (xs[0].bc || xs[1].bc) face_ghost<GAS, S, N, true, T>(a, i0, j0, xs);
                if (ys[0].bc || ys[1].bc) face_ghost<GAS, S, N, false, T>(a, i0, j0, ys);
                S Fx[4], Fy[4];
                unsigned bad = 0;
                riemann_rec<RIEM>(xs[0].R, xs[1].R, xs[0].nx, xs[0].ny, Fx, MathDeferred{bad});
                riemann_rec<RIEM>(ys[0].R, ys[1].R, ys[0].nx, ys[0].ny, Fy, MathDeferred{bad});
                face_jumps<S, N, GEO, true, T>(a, i0, j0, vx, xs, Fx, sF, sG, sDel);
                face_jumps<S, N, GEO, false, T>(a, i0, j0, vy, ys, Fy, sF, sG, sDel);
                if (bad)
                {
                    if (vx) face_point(XFace{}, t, t < NXF, MathChecked{});
                    if (vy) face_point(YFace{}, t, t < NYF, MathChecked{});
                }
            }
            else if (t - PFP < NCOL)
                column(t - PFP);
        }
    }
    __syncthreads();
    // tensor cores: the eta-derivatives of line t (element column k = l of set 1, and of
    // set 3 on curved meshes) go to sC at the nodes (m, l), as the column pass stores them
    float xiF[8], xiG[8];
    if constexpr (TC)
    {
        static_assert(UNPAIR, "the column warps pack the second pass");
        // phase 1: pass 1's MMAs (issued after phase 0 completed) are done
        const bool done = tc::mbar_wait(tc_bar, 1, 1 << 20);
        tc::fence_after_sync();
        if (!done && tid == 0 && a.bad) atomicAdd(a.bad, 1ull << 32);  // flagged, never waited on again
        const int t = tid, eq = t % 4, l = (t / 4) % N, e = t / (4 * N);
        const uint32_t tile = uint32_t(t / tc::kTileLines);
        constexpr uint32_t P1 = 2 * T::LSP * tc::kCols;  // first column of pass 1
        float dG[8], dF[8];
        tc::load8(tmem, P1 + tile * tc::kCols, dG);
        if constexpr (GEO == GEO_CURVED) tc::load8(tmem, P1 + (2 + tile) * tc::kCols, dF);
        tc::load8(tmem, tile * tc::kCols, xiF);
        if constexpr (GEO == GEO_CURVED) tc::load8(tmem, (2 + tile) * tc::kCols, xiG);
        if (t < T::LINES && (e % TX) < txe && (e / TX) < tye)
        {
            if constexpr (GEO == GEO_CURVED)
            {
                const double* mt = a.metrics + ((int64_t(j0 + e / TX + a.row_base) * Nx + (i0 + e % TX)) * NN + l) * 4 + 2;
#pragma unroll
                for (int m = 0; m < N; ++m)
                {
                    const double2 me = __ldg(reinterpret_cast<const double2*>(mt + m * N * 4));
                    sC[(e * 4 + eq) * NN + m * N + l] = R_t(me.x) * dF[m] + R_t(me.y) * dG[m];
                }
            }
            else
            {
#pragma unroll
                for (int m = 0; m < N; ++m) sC[(e * 4 + eq) * NN + m * N + l] = R_t(a.eta_y) * dG[m];
            }
        }
        __syncthreads();
    }

    // ---- P3: element rows (e, eq, l), equation fastest across lanes
    for (int t = tid; t < TE * 4 * N; t += BT)
    {
        const int eq = t % 4, l = (t / 4) % N, e = t / (4 * N);
        const int tx = e % TX, ty = e / TX;
        if (tx >= txe || ty >= tye) continue;
        const S* Fr = sF + (e * 4 + eq) * NN + l * N;
        S fv[N];
        if constexpr (!TC)
        {
#pragma unroll
            for (int m = 0; m < N; ++m) fv[m] = Fr[m];
            center_line<S, N>(fv);
        }
        const R_t dLl = opL<R_t>(ops, l), dRl = opR<R_t>(ops, l);
        const S dxl = sDel[((e * 4 + 0) * 4 + eq) * N + l];
        const S dxr = sDel[((e * 4 + 1) * 4 + eq) * N + l];
        const S* dyb = sDel + ((e * 4 + 2) * 4 + eq) * N;
        const S* dyt = sDel + ((e * 4 + 3) * 4 + eq) * N;
        const int64_t gbase = (int64_t(j0 + ty) * Nx + (i0 + tx)) * ND + eq;
        // coloured Jacobian: this slice's column d of the blocks of colour-c elements
        const int jz = int(blockIdx.z), jc = jz / ND, jd = jz % ND;
        const int jcol = a.mode == MODE_JAC ? elem_colour(a.jac_cmode, Nx, Ny, a.per_x, a.per_y, i0 + tx, j0 + ty) : 0;
        const bool jac_store = a.mode == MODE_JAC && (a.jac_cmode == 2 || jcol == jc);
        // distance-2 colouring: the one element of colour jc in this element's face
        // neighbourhood sits in slot (jc - colour) mod 5: 0 self, 1 right, 2 top, 3 bottom, 4 left
        const int64_t jblk = a.jac_cmode == 2
                                 ? (int64_t(j0 + ty) * Nx + (i0 + tx)) * 5 + (jc - jcol + 5) % 5
                                 : (int64_t(j0 + ty) * Nx + (i0 + tx));
        S gr[N];
        if constexpr (GEO == GEO_CURVED && !TC)
        {
            const S* Gr = sG + (e * 4 + eq) * NN + l * N;
#pragma unroll
            for (int m = 0; m < N; ++m) gr[m] = Gr[m];
            center_line<S, N>(gr);
        }
#pragma unroll
        for (int k = 0; k < N; ++k)
        {
            S dF = S(0.0);
            if constexpr (TC)
                dF = xiF[k];
            else
            {
#pragma unroll
                for (int m = 0; m < N; ++m) dF = dF + opD<R_t>(ops, k * N + m) * fv[m];
            }
            S R;
            if constexpr (GEO == GEO_CURVED)
            {
                S dG = S(0.0);
                if constexpr (TC)
                    dG = xiG[k];
                else
                {
#pragma unroll
                    for (int m = 0; m < N; ++m) dG = dG + opD<R_t>(ops, k * N + m) * gr[m];
                }
                const double2 mx = __ldg(reinterpret_cast<const double2*>(
                    a.metrics + ((int64_t(j0 + ty + a.row_base) * Nx + (i0 + tx)) * NN + l * N + k) * 4));
                R = (R_t(mx.x) * dF + R_t(mx.y) * dG) + sC[(e * 4 + eq) * NN + l * N + k];
            }
            else
            {
                const S px = R_t(a.xi_x) * dF;
                R = px + sC[(e * 4 + eq) * NN + l * N + k];
            }
            R = R + dxl * opL<R_t>(ops, k);
            R = R + dxr * opR<R_t>(ops, k);
            R = R + dyb[k] * dLl;
            R = R + dyt[k] * dRl;
            const int64_t gidx = gbase + (l * N + k) * 4;
            double* out = reinterpret_cast<double*>(a.out);
            if constexpr (T::JVP)
            {
                double jv = a.sigma * sSeed[(e * 4 + eq) * NN + l * N + k] * a.inv_h;
                jv += s_im(R) * a.inv_h;
                if (a.mode != MODE_JAC) out[gidx] = jv;
                else if (jac_store)
                    out[jblk * int64_t(ND * ND) + int64_t(jd) * ND + (l * N + k) * 4 + eq] = jv;
            }
            else if (a.out_f32)
                reinterpret_cast<float*>(a.out)[gidx] = static_cast<float>(s_re(R));
            else if (post)
            {
                // the epilogue's input; without the filter the value is also final
                // unless the limiter changes its element, so it is stored now
                const double v = stage_value(a.st, gidx, s_re(R));
                sO[e * ND + (l * N + k) * 4 + eq] = v;
                if (!(a.post & POST_FILTER)) out[gidx] = v;
            }
            else
            {
                store_residual(a.mode, a.W, a.st, out, gidx, s_re(R));
            }
        }
    }
    if constexpr (TC)
    {
        // every tcgen05.ld of the CTA is complete: warp 0 frees the columns
        tc::fence_before_sync();
        __syncthreads();
        if (tid < 32)
        {
            tc::fence_after_sync();
            tc::tmem_free(tmem, T::TC_COLS);
        }
    }
    if constexpr (post)
    {
        if constexpr (!TC) __syncthreads();
        stage_epilogue<T, N, GAS>(a, ops, i0, j0, txe, tye, sO, base);
    }
}

template <class S, int N, int GAS, int RIEM, int GEO, bool POST, bool TC>
__global__ void __launch_bounds__((Tile2D<S, N, GEO, 0, TC>::BT)) __maxnreg__((Tile2D<S, N, GEO, 0, TC>::MAXREG))
fr2d_kernel(const __grid_constant__ Fr2dArgs a)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    fr2d_tile<S, N, GAS, RIEM, GEO, 0, POST, TC>(a, a.ops, blockIdx.x, blockIdx.y, smem_raw);
}

template <class S, int N, int GAS, int RIEM, int GEO, bool POST, bool TC = false>
cudaError_t launch_fr2d_kernel_v(const Fr2dArgs& a, cudaStream_t st)
{
    using T = Tile2D<S, N, GEO, 0, TC>;
    auto kern = fr2d_kernel<S, N, GAS, RIEM, GEO, POST, TC>;
    constexpr size_t bytes = POST ? T::bytes_post : T::bytes_launch;
    // kernel attributes are per device: set them once on each device that launches
    static bool attr_done[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64 || !attr_done[dev])
    {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) attr_done[dev] = true;
    }
    dim3 grid((a.Nx + T::TX - 1) / T::TX, (a.row_end - a.row_begin + T::TY - 1) / T::TY,
              a.mode == MODE_JAC ? (a.jac_cmode == 2 ? 5 : a.jac_cmode ? 9 : 2) * T::NN * 4 : 1);
    kern<<<grid, T::BT, bytes, st>>>(a);
    return cudaGetLastError();
}

template <class S, int N, int GAS, int RIEM, int GEO>
cudaError_t launch_fr2d_kernel(const Fr2dArgs& a, cudaStream_t st)
{
    if constexpr (sizeof(S) == 4 && N >= 5 && N <= 8)
    {
        // the FP32 tiles with their derivative contractions on the tensor cores
        if (a.tc && a.mode != MODE_JAC)
        {
            if (a.mode == MODE_STAGE && a.post) return launch_fr2d_kernel_v<S, N, GAS, RIEM, GEO, true, true>(a, st);
            return launch_fr2d_kernel_v<S, N, GAS, RIEM, GEO, false, true>(a, st);
        }
    }
    if constexpr (scalar_traits<S>::words == 1)
    {
        if (a.mode == MODE_STAGE && a.post) return launch_fr2d_kernel_v<S, N, GAS, RIEM, GEO, true>(a, st);
    }
    return launch_fr2d_kernel_v<S, N, GAS, RIEM, GEO, false>(a, st);
}

// ---- batches ------------------------------------------------------------------
// Stage k of SSP-RK3 (Shu and Osher) for instance `in` at its own clock, in the form the
// integrator's stages take (fr_sdg_b200/integrate.py):
//   k = 0: b0 = U + h L(U);  k = 1: b1 = 3/4 U + 1/4 b0 + h/4 L(b0);
//   k = 2: b2 = 1/3 U + 2/3 b1 + 2h/3 L(b1).
// The mixed form (FP32 instantiation) reads the same FP64 stage inputs and recovers
// every node's primitives in FP64 (Fr2dArgs::in_f64).  Each stage output passes the
// instance's stage epilogue (post[k]); with fused_step the last one is the whole
// post-step and the stage writes the state itself.
__device__ __forceinline__ void batch_stage_args(Fr2dArgs& a, const BatchInst2D& in, const BatchClock& ck, int k,
                                                 bool mixed)
{
    const double h = batch_step_size(ck);
    a.mode = MODE_STAGE;
    a.cond_sys = 0;
    a.out_f32 = 0;
    a.in_f64 = mixed ? 1 : 0;
    a.W = nullptr;
    a.st.acc = nullptr;
    a.st.delta = 0.0;
    a.st.out32 = nullptr;
    a.st.A = in.U;
    a.post = in.post[k];
    a.pa = in.pa;
    if (k == 0)
    {
        a.U = in.U;
        a.out = in.b[0];
        a.st.B = nullptr;
        a.st.alpha = 1.0;
        a.st.beta = 0.0;
        a.st.gamma = h;
        a.t = ck.t;
    }
    else if (k == 1)
    {
        a.U = in.b[0];
        a.out = in.b[1];
        a.st.B = in.b[0];
        a.st.alpha = 0.75;
        a.st.beta = 0.25;
        a.st.gamma = 0.25 * h;
        a.t = ck.t + h;
    }
    else
    {
        a.U = in.b[1];
        a.out = in.fused_step ? in.U : in.b[2];
        a.st.B = in.b[1];
        a.st.alpha = 1.0 / 3.0;
        a.st.beta = 2.0 / 3.0;
        a.st.gamma = 2.0 * h / 3.0;
        a.t = ck.t + 0.5 * h;
    }
}

// One SSP-RK3 stage of a batch group: persistent CTAs walk the group's tile list
// (instance in group, bx, by), copy the instance's launch arguments (all but the
// operators, which are the group's) into shared memory and run the residual tile with
// the stage epilogue.  Inactive instances (clock) are skipped.
template <class S, int N, int GAS, int RIEM, int VAR, bool POST>
__global__ void __launch_bounds__((Tile2D<S, N, GEO_AFFINE, VAR>::BT)) __maxnreg__((Tile2D<S, N, GEO_AFFINE, VAR>::MAXREG))
fr2d_batch_kernel(const __grid_constant__ Fr2dBatchArgs b)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(16) unsigned long long sa_raw[(sizeof(Fr2dArgs) + 7) / 8];
    Fr2dArgs& sa = *reinterpret_cast<Fr2dArgs*>(sa_raw);
    constexpr int HEAD = int(offsetof(Fr2dArgs, ops) / 8);  // the arguments before the operators
    for (int tile = blockIdx.x; tile < b.ntiles; tile += gridDim.x)
    {
        const int4 tm = b.tiles[tile];
        const BatchInst2D& in = b.inst[tm.x];
        const BatchClock ck = b.clock[in.inst];
        if (!ck.active) continue;  // uniform over the CTA
        __syncthreads();           // the previous tile is done with sa and the tile memory
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&in.a);
        for (int q = threadIdx.x; q < HEAD; q += blockDim.x) sa_raw[q] = src[q];
        __syncthreads();
        if (threadIdx.x == 0) batch_stage_args(sa, in, ck, b.stage, b.mixed != 0);
        __syncthreads();
        fr2d_tile<S, N, GAS, RIEM, GEO_AFFINE, VAR, POST>(sa, b.ops, tm.y, tm.z, smem_raw);
    }
}

// POST: the instantiation with the stage epilogue, for the stage that carries a post-step
// (the last); the others skip the epilogue's registers and spills.
template <class S, int N, int GAS, int RIEM, int VAR, bool POST>
cudaError_t launch_fr2d_batch_kernel_v(const Fr2dBatchArgs& b, int grid, cudaStream_t st, int* occupancy)
{
    using T = Tile2D<S, N, GEO_AFFINE, VAR>;
    auto kern = fr2d_batch_kernel<S, N, GAS, RIEM, VAR, POST>;
    constexpr size_t bytes = POST ? T::bytes_post : T::bytes_launch;
    static bool attr_done[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64 || !attr_done[dev])
    {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) attr_done[dev] = true;
    }
    if (occupancy) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occupancy, kern, T::BT, bytes);
    if (grid > 0 && b.ntiles > 0) kern<<<grid, T::BT, bytes, st>>>(b);
    return cudaGetLastError();
}

template <class S, int N, int GAS, int RIEM, int VAR>
cudaError_t launch_fr2d_batch_kernel(const Fr2dBatchArgs& b, int grid, cudaStream_t st, int* occupancy)
{
    if (b.stage == 2) return launch_fr2d_batch_kernel_v<S, N, GAS, RIEM, VAR, true>(b, grid, st, occupancy);
    return launch_fr2d_batch_kernel_v<S, N, GAS, RIEM, VAR, false>(b, grid, st, occupancy);
}

// Batched stage launcher of one order N (affine geometry): grid CTAs, or with
// `occupancy` set only the number of CTAs of the variant that fit on one SM.
template <class S, int N>
cudaError_t launch_fr2d_batch(int gas, int riem, int var, const Fr2dBatchArgs& b, int grid, cudaStream_t s,
                              int* occupancy)
{
    const int key = (gas * 2 + riem) * 2 + (var ? 1 : 0);
    switch (key)
    {
        case 0: return launch_fr2d_batch_kernel<S, N, 0, 0, 0>(b, grid, s, occupancy);
        case 1: return launch_fr2d_batch_kernel<S, N, 0, 0, 1>(b, grid, s, occupancy);
        case 2: return launch_fr2d_batch_kernel<S, N, 0, 1, 0>(b, grid, s, occupancy);
        case 3: return launch_fr2d_batch_kernel<S, N, 0, 1, 1>(b, grid, s, occupancy);
        case 4: return launch_fr2d_batch_kernel<S, N, 1, 0, 0>(b, grid, s, occupancy);
        case 5: return launch_fr2d_batch_kernel<S, N, 1, 0, 1>(b, grid, s, occupancy);
        case 6: return launch_fr2d_batch_kernel<S, N, 1, 1, 0>(b, grid, s, occupancy);
        case 7: return launch_fr2d_batch_kernel<S, N, 1, 1, 1>(b, grid, s, occupancy);
        default: return cudaErrorInvalidValue;
    }
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
