// batch.cu -- frsdg_batch: many independent 2D instances advanced together to their own
// final times (the batched workload of many small problems).
//
// Instances that share the order, the gas law, the Riemann solver and the VCJH
// correction form a group.  One SSP-RK3 step of the whole batch is a fixed sequence
// of launches:
//   for each stage k: one residual+stage launch per group over the concatenated tiles
//     of its instances (persistent CTAs walking a tile list, batch_stage_args),
//     then the positivity limiter of that stage's output (one launch per group);
//   the post-step stabilisation of the last stage into the state (one launch per
//     group), the limiter of the state, and the clock kernel.
// Every instance keeps its own time step and final time on the device (BatchClock), so
// the step needs no host input: frsdg_batch_run captures it once into a CUDA graph and
// replays that graph until every instance has reached its final time.  An autotuner
// picks, per group, the tile (elements per CTA) and the number of persistent CTAs by
// timing the candidates' stage launches with CUDA events, and caches the choice.
#include "handle.hpp"
#include "frsdg_internal.hpp"
#include "pplimit.hpp"
#include "stab.hpp"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

using namespace frsdg;

namespace frsdg
{
int report(int code, const char* msg);
int report_cuda(cudaError_t e, const char* what);
} // namespace frsdg

namespace
{

template <class S>
cudaError_t stage_launch(int n, int gas, int riem, int var, const Fr2dBatchArgs& a, int grid, cudaStream_t s, int* occ)
{
    switch (n)
    {
        case 2: return launch_fr2d_batch<S, 2>(gas, riem, var, a, grid, s, occ);
        case 3: return launch_fr2d_batch<S, 3>(gas, riem, var, a, grid, s, occ);
        case 4: return launch_fr2d_batch<S, 4>(gas, riem, var, a, grid, s, occ);
        case 5: return launch_fr2d_batch<S, 5>(gas, riem, var, a, grid, s, occ);
        case 6: return launch_fr2d_batch<S, 6>(gas, riem, var, a, grid, s, occ);
        case 7: return launch_fr2d_batch<S, 7>(gas, riem, var, a, grid, s, occ);
        case 8: return launch_fr2d_batch<S, 8>(gas, riem, var, a, grid, s, occ);
        case 9: return launch_fr2d_batch<S, 9>(gas, riem, var, a, grid, s, occ);
        case 10: return launch_fr2d_batch<S, 10>(gas, riem, var, a, grid, s, occ);
        default: return cudaErrorInvalidValue;
    }
}

// Tile of the batched residual (elements along x, y) for one order, scalar and variant:
// the tile_x / tile_y shapes of the single-instance kernel, variant 1 with half the rows.
void residual_tile(int n, bool f32, int var, int* tx, int* ty)
{
    *tx = tile_x(n, 1, f32);
    const int t = tile_y(n, 1, f32);
    *ty = var == 0 || t == 1 ? t : t / 2;
}

// Autotuner choices, per (device, order, gas, flux, precision, tile count rounded up to a
// power of two).
struct TuneKey
{
    int dev, n, gas, riem, mixed, tiles_pow2;
    bool operator<(const TuneKey& o) const
    {
        return std::tie(dev, n, gas, riem, mixed, tiles_pow2) < std::tie(o.dev, o.n, o.gas, o.riem, o.mixed, o.tiles_pow2);
    }
};
struct TuneChoice
{
    int var, grid_mult;
    float ms;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneChoice> g_tune_cache;

struct Group
{
    int    n = 0, gas = 0, riem = 0;
    double radau = 0.0;
    std::vector<int> members;  // batch indices
    Ops    ops{};
    BatchInst2D* d_inst = nullptr;
    int4*  d_tiles[2] = {nullptr, nullptr};
    int    ntiles[2] = {0, 0};
    std::vector<int4> h_tiles[2];  // host copies (pruned as instances finish)
    int    occ = 0;                // resident CTAs per SM of the chosen variant
    StabArgs* d_stab = nullptr;
    int*   d_stab_clock = nullptr;
    int4*  d_stab_tiles = nullptr;
    int    nstab = 0;              // post-step tiles of the instances whose post-step is not fused
    int    unfused = 0;            // such instances
    int    any_pp = 0;             // instances with the positivity limiter
    PPArgs* d_pp = nullptr;
    int64_t* d_elem_begin = nullptr;
    int64_t nelem = 0;
    int    var = 0, grid = 0;  // autotuner's choice (grid: persistent CTAs of the stage launch)
    int    grid_mult = 0;
    float  tuned_ms = 0.0f;
};

} // namespace

struct frsdg_batch
{
    int count = 0, mixed = 0, device = 0, sm_count = 0;
    std::vector<frsdg_handle*> handles;
    std::vector<Group> groups;
    BatchClock* d_clock = nullptr;
    PostArgs* d_post = nullptr;  // stage-epilogue operands per instance
    int*   d_active = nullptr;
    int*   h_active = nullptr;  // pinned
    std::vector<void*> allocs;
    bool   tuned = false;
    cudaStream_t cs = nullptr;  // the batch's own stream (graph capture and replay)
    cudaGraphExec_t exec = nullptr;
    int    live = 0;            // instances active when the graph was captured
    cudaEvent_t ev[2] = {nullptr, nullptr};
};

namespace
{

void free_batch(frsdg_batch* b)
{
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    for (auto& g : b->groups)
    {
        cudaFree(g.d_inst);
        cudaFree(g.d_tiles[0]);
        cudaFree(g.d_tiles[1]);
        cudaFree(g.d_stab);
        cudaFree(g.d_stab_clock);
        cudaFree(g.d_stab_tiles);
        cudaFree(g.d_pp);
        cudaFree(g.d_elem_begin);
    }
    for (void* p : b->allocs) cudaFree(p);
    cudaFree(b->d_clock);
    cudaFree(b->d_post);
    cudaFree(b->d_active);
    if (b->h_active) cudaFreeHost(b->h_active);
    for (cudaEvent_t& e : b->ev)
        if (e) cudaEventDestroy(e);
    if (b->cs) cudaStreamDestroy(b->cs);
    delete b;
}

template <class T> cudaError_t upload(T** dst, const std::vector<T>& v)
{
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(dst), sizeof(T) * (v.empty() ? 1 : v.size()));
    if (e != cudaSuccess || v.empty()) return e;
    return cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice);
}

Fr2dBatchArgs stage_args(const frsdg_batch* b, const Group& g, int var, int k)
{
    Fr2dBatchArgs a{};
    a.ops = g.ops;
    a.inst = g.d_inst;
    a.clock = b->d_clock;
    a.tiles = g.d_tiles[var];
    a.ntiles = g.ntiles[var];
    a.stage = k;
    a.mixed = b->mixed;
    return a;
}

cudaError_t launch_stage(const frsdg_batch* b, const Group& g, int var, int grid, int k, cudaStream_t s)
{
    const Fr2dBatchArgs a = stage_args(b, g, var, k);
    return b->mixed ? stage_launch<float>(g.n, g.gas, g.riem, var, a, grid, s, nullptr)
                    : stage_launch<double>(g.n, g.gas, g.riem, var, a, grid, s, nullptr);
}

cudaError_t launch_pp(const frsdg_batch* b, const Group& g, int slot, cudaStream_t s)
{
    PPBatchArgs p{};
    p.inst = g.d_pp;
    p.binst = g.d_inst;
    p.elem_begin = g.d_elem_begin;
    p.ninst = int(g.members.size());
    p.nelem = g.nelem;
    p.clock = b->d_clock;
    p.slot = slot;
    return launch_pp_batch(g.n, p, s);
}

// One SSP-RK3 step of every active instance, enqueued on s: per stage one launch per
// group and the limiter pass; for instances with an element-local post-step (the
// filter, the limiter) the last stage's epilogue is the whole post-step, yields the
// wave speed and writes the state.  The WENO post-step of the others follows as its
// own pass, then their limiter and wave speeds.
cudaError_t enqueue_step(const frsdg_batch* b, cudaStream_t s)
{
    cudaError_t e;
    for (int k = 0; k < 3; ++k)
    {
        for (const Group& g : b->groups)
            if ((e = launch_stage(b, g, g.var, g.grid, k, s)) != cudaSuccess) return e;
        for (const Group& g : b->groups)
            if ((k < 2 ? g.any_pp : g.unfused) && (e = launch_pp(b, g, k, s)) != cudaSuccess) return e;
    }
    for (const Group& g : b->groups)
    {
        if (!g.nstab) continue;
        StabBatchArgs sb{g.d_stab, g.d_stab_clock, b->d_clock, g.d_stab_tiles, g.nstab};
        if ((e = launch_stab_batch(g.n, sb, s)) != cudaSuccess) return e;
    }
    for (const Group& g : b->groups)
        if (g.unfused && (e = launch_pp(b, g, 3, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(b->d_active, 0, sizeof(int), s)) != cudaSuccess) return e;
    return launch_batch_clock(b->d_clock, b->count, b->d_active, s);
}

// Time one stage launch of a candidate (mean of three after one warm-up).
float time_candidate(const frsdg_batch* b, const Group& g, int var, int grid, cudaStream_t s)
{
    if (launch_stage(b, g, var, grid, 0, s) != cudaSuccess) return 1e30f;
    cudaEventRecord(b->ev[0], s);
    for (int r = 0; r < 3; ++r)
        if (launch_stage(b, g, var, grid, 0, s) != cudaSuccess) return 1e30f;
    cudaEventRecord(b->ev[1], s);
    if (cudaEventSynchronize(b->ev[1]) != cudaSuccess) return 1e30f;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]);
    return ms / 3.0f;
}

// Candidates: tile variant 0 / 1 (half the element rows per CTA), and one CTA per tile
// or 1, 2, 4 resident waves of persistent CTAs.  Stage 0 only reads the state and writes
// the first stage buffer, so timing it changes nothing.
int autotune(frsdg_batch* b, cudaStream_t s)
{
    for (Group& g : b->groups)
    {
        const int p2 = [&] {
            int v = 1;
            while (v < g.ntiles[0]) v <<= 1;
            return v;
        }();
        const TuneKey key{b->device, g.n, g.gas, g.riem, b->mixed, p2};
        bool cached = false;
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            auto it = g_tune_cache.find(key);
            if (it != g_tune_cache.end())
            {
                g.var = it->second.var;
                g.grid_mult = it->second.grid_mult;
                g.tuned_ms = it->second.ms;
                cached = true;
            }
        }
        if (!cached)
        {
            float best = 1e30f;
            for (int var = 0; var < 2; ++var)
            {
                if (var == 1)
                {
                    int tx0, ty0, tx1, ty1;
                    residual_tile(g.n, b->mixed != 0, 0, &tx0, &ty0);
                    residual_tile(g.n, b->mixed != 0, 1, &tx1, &ty1);
                    if (ty1 == ty0) continue;  // no second shape at this order
                }
                int occ = 0;
                const Fr2dBatchArgs a = stage_args(b, g, var, 0);
                const cudaError_t e = b->mixed ? stage_launch<float>(g.n, g.gas, g.riem, var, a, 0, s, &occ)
                                               : stage_launch<double>(g.n, g.gas, g.riem, var, a, 0, s, &occ);
                if (e != cudaSuccess) return report_cuda(e, "batch autotuner: occupancy");
                for (int mult : {0, 1, 2, 4})
                {
                    const int grid = mult == 0 ? g.ntiles[var] : std::min(g.ntiles[var], mult * std::max(occ, 1) * b->sm_count);
                    const float ms = time_candidate(b, g, var, grid, s);
                    if (ms < best)
                    {
                        best = ms;
                        g.var = var;
                        g.grid_mult = mult;
                        g.tuned_ms = ms;
                    }
                }
            }
            if (best >= 1e30f) return report(FRSDG_ERR_CUDA, "batch autotuner: no candidate ran");
            std::lock_guard<std::mutex> lk(g_tune_mu);
            g_tune_cache[key] = TuneChoice{g.var, g.grid_mult, g.tuned_ms};
        }
        int occ = 0;
        const Fr2dBatchArgs a = stage_args(b, g, g.var, 0);
        const cudaError_t e = b->mixed ? stage_launch<float>(g.n, g.gas, g.riem, g.var, a, 0, s, &occ)
                                       : stage_launch<double>(g.n, g.gas, g.riem, g.var, a, 0, s, &occ);
        if (e != cudaSuccess) return report_cuda(e, "batch autotuner: occupancy");
        g.occ = occ;
        g.grid = g.grid_mult == 0 ? g.ntiles[g.var]
                                  : std::min(g.ntiles[g.var], g.grid_mult * std::max(occ, 1) * b->sm_count);
    }
    b->tuned = true;
    return FRSDG_OK;
}

// Drop the tiles of finished instances from every group's stage tile list (the
// persistent CTAs otherwise keep walking them) and forget the captured step, which
// holds the old counts.  Called between replays, with the batch stream idle.
int prune(frsdg_batch* b)
{
    std::vector<BatchClock> clk(static_cast<size_t>(b->count));
    cudaError_t e = cudaMemcpy(clk.data(), b->d_clock, sizeof(BatchClock) * clk.size(), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return report_cuda(e, "batch clocks");
    int live = 0;
    for (const BatchClock& c : clk) live += c.active ? 1 : 0;
    for (Group& g : b->groups)
    {
        std::vector<int4>& ht = g.h_tiles[g.var];
        std::vector<int4> keep;
        keep.reserve(ht.size());
        for (const int4& t : ht)
            if (clk[size_t(g.members[size_t(t.x)])].active) keep.push_back(t);
        if (keep.size() == ht.size()) continue;
        ht.swap(keep);
        if (!ht.empty() &&
            (e = cudaMemcpy(g.d_tiles[g.var], ht.data(), sizeof(int4) * ht.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
            return report_cuda(e, "batch tiles");
        g.ntiles[g.var] = int(ht.size());
        g.grid = g.grid_mult == 0 ? g.ntiles[g.var]
                                  : std::min(g.ntiles[g.var], g.grid_mult * std::max(g.occ, 1) * b->sm_count);
    }
    if (b->exec)
    {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    b->live = live;
    return FRSDG_OK;
}

} // namespace

extern "C" {

int frsdg_batch_create(frsdg_handle* const* handles, int32_t count, double* const* states, const double* dt,
                       const double* dt_scale, const double* t_end, int32_t mixed, frsdg_batch** out)
{
    if (!handles || !states || !dt || !t_end || !out || count <= 0) return report(FRSDG_ERR_ARG, "null argument");
    *out = nullptr;
    for (int i = 0; i < count; ++i)
    {
        const frsdg_handle* h = handles[i];
        if (!h || !states[i]) return report(FRSDG_ERR_ARG, "null handle or state");
        if (h->cfg.dim != 2 || h->geo != GEO_AFFINE || h->win_rows || h->cfg.cond_sys)
            return report(FRSDG_ERR_UNSUPPORTED,
                          "frsdg_batch: 2D affine instances without row window or change of variables only");
        if (reinterpret_cast<uintptr_t>(states[i]) & 15) return report(FRSDG_ERR_ARG, "states must be 16-byte aligned");
        if (!(dt[i] > 0.0)) return report(FRSDG_ERR_ARG, "dt must be positive");
    }
    auto* b = new frsdg_batch();
    b->count = count;
    b->mixed = mixed ? 1 : 0;
    b->handles.assign(handles, handles + count);
    cudaError_t e;
    auto fail_cuda = [&](cudaError_t err, const char* what) {
        free_batch(b);
        return report_cuda(err, what);
    };
    if ((e = cudaGetDevice(&b->device)) != cudaSuccess) return fail_cuda(e, "cudaGetDevice");
    if ((e = cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, b->device)) != cudaSuccess)
        return fail_cuda(e, "device attribute");
    // groups by (order, gas law, flux, correction, filter): the group's operators
    std::map<std::tuple<int, int, int, double, int, int, double>, int> gid;
    for (int i = 0; i < count; ++i)
    {
        const frsdg_handle* h = handles[i];
        const auto key = std::make_tuple(h->n, h->cfg.gas_law, h->cfg.riemann, h->cfg.radau_corr, h->cfg.filt_cut_off,
                                         h->cfg.filt_strength, h->cfg.filt_alpha);
        auto it = gid.find(key);
        if (it == gid.end())
        {
            it = gid.emplace(key, int(b->groups.size())).first;
            Group g;
            g.n = h->n;
            g.gas = h->cfg.gas_law;
            g.riem = h->cfg.riemann;
            g.radau = h->cfg.radau_corr;
            g.ops = h->a2.ops;
            b->groups.push_back(g);
        }
        b->groups[size_t(it->second)].members.push_back(i);
    }
    // clocks
    std::vector<BatchClock> clk(static_cast<size_t>(count));
    for (int i = 0; i < count; ++i)
        clk[size_t(i)] = BatchClock{0.0, dt[i], t_end[i], 1, dt_scale ? 1 : 0, dt_scale ? dt_scale[i] : 0.0, 0ull, 0ll,
                                    1e-3 * dt[i]};
    if ((e = upload(&b->d_clock, clk)) != cudaSuccess) return fail_cuda(e, "batch clocks");
    // stage-epilogue operands: the handle's filter, weights and floor, and the clock's
    // wave-speed slot for adaptive steps
    std::vector<PostArgs> post(static_cast<size_t>(count));
    for (int i = 0; i < count; ++i)
    {
        const frsdg_handle* h = handles[i];
        PostArgs& p = post[size_t(i)];
        for (int q = 0; q < h->n; ++q) p.w[q] = h->re.w[q];
        p.pp_eps = h->cfg.pp_eps;
        p.detJ = nullptr;  // affine
        p.amax = dt_scale ? &b->d_clock[i].amax : nullptr;
    }
    if ((e = upload(&b->d_post, post)) != cudaSuccess) return fail_cuda(e, "batch epilogue operands");
    if ((e = cudaMalloc(&b->d_active, sizeof(int))) != cudaSuccess) return fail_cuda(e, "batch counter");
    if ((e = cudaMallocHost(&b->h_active, sizeof(int))) != cudaSuccess) return fail_cuda(e, "batch counter");
    for (Group& g : b->groups)
    {
        std::vector<BatchInst2D> inst;
        std::vector<StabArgs> stab;
        std::vector<int> stab_clock;
        std::vector<PPArgs> pp;
        std::vector<int64_t> elem_begin{0};
        std::vector<int4> tiles[2], stiles;
        int stx, sty;
        stab_tile_dims(g.n, &stx, &sty);
        for (size_t m = 0; m < g.members.size(); ++m)
        {
            const int i = g.members[m];
            frsdg_handle* h = handles[i];
            BatchInst2D in{};
            in.a = h->a2;
            in.U = states[i];
            in.inst = i;
            in.pa = b->d_post + i;
            // stage epilogues: the limiter on every stage output; the last stage also
            // runs an element-local post-step (filter) and yields the wave speed
            const bool pp_on = h->cfg.pp_limit != 0;
            const bool fused = h->cfg.apply_filter || !h->cfg.apply_weno;
            // (the first two stages' limiter runs as its own pass: measured faster than
            // the epilogue on the 1024^2 p = 5 blast, 2.44 against 2.70 ms per stage)
            in.post[0] = in.post[1] = 0;
            in.fused_step = fused ? 1 : 0;
            in.post[2] = fused ? (pp_on ? POST_PP : 0) | (h->cfg.apply_filter ? POST_FILTER : 0) |
                                     (dt_scale ? POST_AMAX : 0)
                               : 0;
            if (pp_on) g.any_pp = 1;
            const size_t nt = size_t(h->ntot);
            for (int k = 0; k < 3; ++k)
            {
                void* p = nullptr;
                if ((e = cudaMalloc(&p, sizeof(double) * nt)) != cudaSuccess) return fail_cuda(e, "batch stage buffers");
                b->allocs.push_back(p);
                in.b[k] = static_cast<double*>(p);
            }
            inst.push_back(in);
            StabArgs sa = h->st;
            sa.src = in.b[2];
            sa.dst = in.U;
            stab.push_back(sa);
            stab_clock.push_back(i);
            PPArgs pa = h->pp;
            pa.nelem = h->nelem;
            pa.row_base = 0;
            pa.U = in.U;
            pa.U32 = nullptr;
            pa.fused = fused ? 1 : 0;
            pp.push_back(pa);
            if (!fused) ++g.unfused;
            elem_begin.push_back(elem_begin.back() + h->nelem);
            for (int var = 0; var < 2; ++var)
            {
                int tx, ty;
                residual_tile(g.n, b->mixed != 0, var, &tx, &ty);
                for (int by = 0; by < (h->Ny + ty - 1) / ty; ++by)
                    for (int bx = 0; bx < (h->Nx + tx - 1) / tx; ++bx) tiles[var].push_back(make_int4(int(m), bx, by, 0));
            }
            if (!fused)
                for (int by = 0; by < (h->Ny + sty - 1) / sty; ++by)
                    for (int bx = 0; bx < (h->Nx + stx - 1) / stx; ++bx)
                        stiles.push_back(make_int4(int(m), bx, by, 0));
        }
        g.nelem = elem_begin.back();
        g.ntiles[0] = int(tiles[0].size());
        g.ntiles[1] = int(tiles[1].size());
        g.h_tiles[0] = tiles[0];
        g.h_tiles[1] = tiles[1];
        g.nstab = int(stiles.size());
        if ((e = upload(&g.d_inst, inst)) || (e = upload(&g.d_tiles[0], tiles[0])) || (e = upload(&g.d_tiles[1], tiles[1])) ||
            (e = upload(&g.d_stab, stab)) || (e = upload(&g.d_stab_clock, stab_clock)) ||
            (e = upload(&g.d_stab_tiles, stiles)) || (e = upload(&g.d_pp, pp)) || (e = upload(&g.d_elem_begin, elem_begin)))
            return fail_cuda(e, "batch tables");
    }
    if ((e = cudaStreamCreateWithFlags(&b->cs, cudaStreamNonBlocking)) != cudaSuccess) return fail_cuda(e, "stream");
    for (cudaEvent_t& ev : b->ev)
        if ((e = cudaEventCreate(&ev)) != cudaSuccess) return fail_cuda(e, "events");
    *out = b;
    return FRSDG_OK;
}

int frsdg_batch_destroy(frsdg_batch* b)
{
    free_batch(b);
    return FRSDG_OK;
}

int frsdg_batch_step(frsdg_batch* b, void* stream)
{
    if (!b) return report(FRSDG_ERR_ARG, "null argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!b->tuned)
    {
        const int rc = autotune(b, s);
        if (rc) return rc;
    }
    const cudaError_t e = enqueue_step(b, s);
    if (e != cudaSuccess) return report_cuda(e, "batch step");
    return FRSDG_OK;
}

int frsdg_batch_run(frsdg_batch* b, int64_t max_steps, int64_t* steps, void* stream)
{
    if (!b) return report(FRSDG_ERR_ARG, "null argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if ((e = cudaEventRecord(b->ev[0], s)) != cudaSuccess || (e = cudaStreamWaitEvent(b->cs, b->ev[0], 0)) != cudaSuccess)
        return report_cuda(e, "batch stream order");
    if (!b->tuned)
    {
        const int rc = autotune(b, b->cs);
        if (rc) return rc;
    }
    // the step of every group captured once into a CUDA graph and replayed; the graph is
    // captured again after the tile lists lose a quarter of the live instances
    auto capture = [&]() -> int {
        cudaGraph_t graph = nullptr;
        if ((e = cudaStreamBeginCapture(b->cs, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
            return report_cuda(e, "batch graph capture");
        const cudaError_t el = enqueue_step(b, b->cs);
        e = cudaStreamEndCapture(b->cs, &graph);
        if (el != cudaSuccess) return report_cuda(el, "batch graph capture");
        if (e != cudaSuccess) return report_cuda(e, "batch graph capture");
        e = cudaGraphInstantiate(&b->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return report_cuda(e, "batch graph instantiate");
        return FRSDG_OK;
    };
    if (!b->live) b->live = b->count;
    int64_t k = 0;
    constexpr int kCheck = 16;  // replays between reads of the active count
    while (max_steps <= 0 || k < max_steps)
    {
        if (!b->exec)
        {
            const int rc = capture();
            if (rc) return rc;
        }
        const int reps = max_steps > 0 ? int(std::min<int64_t>(kCheck, max_steps - k)) : kCheck;
        for (int r = 0; r < reps; ++r)
            if ((e = cudaGraphLaunch(b->exec, b->cs)) != cudaSuccess) return report_cuda(e, "batch graph launch");
        k += reps;
        if ((e = cudaMemcpyAsync(b->h_active, b->d_active, sizeof(int), cudaMemcpyDeviceToHost, b->cs)) != cudaSuccess ||
            (e = cudaStreamSynchronize(b->cs)) != cudaSuccess)
            return report_cuda(e, "batch active count");
        if (*b->h_active == 0) break;
        if (4 * *b->h_active < 3 * b->live)
        {
            const int rc = prune(b);
            if (rc) return rc;
        }
    }
    if (steps) *steps = k;
    if ((e = cudaEventRecord(b->ev[1], b->cs)) != cudaSuccess || (e = cudaStreamWaitEvent(s, b->ev[1], 0)) != cudaSuccess)
        return report_cuda(e, "batch stream order");
    return FRSDG_OK;
}

int frsdg_batch_times(const frsdg_batch* b, double* t, int32_t* active, int64_t* steps)
{
    if (!b || !t) return report(FRSDG_ERR_ARG, "null argument");
    std::vector<BatchClock> clk(static_cast<size_t>(b->count));
    const cudaError_t e = cudaMemcpy(clk.data(), b->d_clock, sizeof(BatchClock) * clk.size(), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return report_cuda(e, "batch clocks");
    for (int i = 0; i < b->count; ++i)
    {
        t[i] = clk[size_t(i)].t;
        if (active) active[i] = clk[size_t(i)].active;
        if (steps) steps[i] = clk[size_t(i)].steps;
    }
    return FRSDG_OK;
}

int frsdg_batch_tuning(const frsdg_batch* b, int32_t group, int32_t* order, int32_t* variant, int32_t* grid,
                       int32_t* tiles, float* stage_ms)
{
    if (!b || group < 0 || group >= int(b->groups.size())) return report(FRSDG_ERR_ARG, "bad group");
    const Group& g = b->groups[size_t(group)];
    if (order) *order = g.n;
    if (variant) *variant = g.var;
    if (grid) *grid = g.grid;
    if (tiles) *tiles = g.ntiles[g.var];
    if (stage_ms) *stage_ms = g.tuned_ms;
    return FRSDG_OK;
}

int frsdg_batch_groups(const frsdg_batch* b, int32_t* groups)
{
    if (!b || !groups) return report(FRSDG_ERR_ARG, "null argument");
    *groups = int(b->groups.size());
    return FRSDG_OK;
}

} // extern "C"
