// mms_api.cu — host side of the C ABI declared in include/mms.h.
//
// Owns one device-resident domain per context, applies the reference's
// initial state and nucleation-site draws on the host (they are defined by
// glibc rand() streams and must be replayed exactly), and drives the
// per-step kernel sequence of kernels.cu on one CUDA stream.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <array>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <map>
#include <mutex>
#include <type_traits>
#include <string>
#include <sys/time.h>
#include <unordered_map>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "host_setup.h"
#include "mms_internal.h"
#include "sites.h"

using namespace mms;


// Event bracketing of kernel launches for mms_kernel_stats.
struct EventProfiler : mms::Profiler {
    struct Rec {
        int kid;
        cudaEvent_t a, b;
    };
    std::vector<cudaEvent_t> pool;
    std::vector<Rec> pending;
    double total_ms[mms::KID_COUNT] = {};
    uint64_t count[mms::KID_COUNT] = {};
    cudaEvent_t cur = nullptr;
    cudaEvent_t get()
    {
        if (pool.empty()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            return e;
        }
        cudaEvent_t e = pool.back();
        pool.pop_back();
        return e;
    }
    void begin(int kid, void *stream) override
    {
        (void)kid;
        cur = get();
        cudaEventRecord(cur, (cudaStream_t)stream);
    }
    void end(int kid, void *stream) override
    {
        cudaEvent_t e = get();
        cudaEventRecord(e, (cudaStream_t)stream);
        pending.push_back({kid, cur, e});
    }
    // stream must be idle
    void collect()
    {
        for (const Rec &r : pending) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, r.a, r.b);
            total_ms[r.kid] += ms;
            count[r.kid]++;
            pool.push_back(r.a);
            pool.push_back(r.b);
        }
        pending.clear();
    }
    ~EventProfiler()
    {
        for (cudaEvent_t e : pool) cudaEventDestroy(e);
        for (const Rec &r : pending) {
            cudaEventDestroy(r.a);
            cudaEventDestroy(r.b);
        }
    }
};

struct mms_ctx {
    mms_params p{};
    TmaHolder tma{};
    // FP32 AM contraction tile rows: 64-128 (a multiple of 16; two
    // accumulator sets), 256 (one), 0 = 128; set by mms_set_am_tile or
    // mms_autotune
    int am_rows = 0;
    // one timestep captured as a CUDA graph (kernel arguments only change
    // when sites or orientation overrides are replaced)
    cudaGraphExec_t step_graph = nullptr;
    int step_graph_kernels = 0;
    // GRAPH_STEPS consecutive steps in one graph (fewer graph boundaries)
    cudaGraphExec_t multi_graph = nullptr;
    // one step whose stencil also leaves its per-tile fraction-solid sums
    // (the last step of mms_step_reduce)
    cudaGraphExec_t sum_graph = nullptr;
    bool use_graphs = true;
    cudaStream_t own_stream = nullptr;
    EventProfiler *prof = nullptr;
    std::vector<mms_fixed_nuc> fixed;
    std::vector<mms_nuc_volume> vols;
    int prec = MMS_PREC_F64;
    int device = 0;
    cudaStream_t stream = nullptr;
    KernelArgs ka{};
    std::vector<Rank> ranks;
    // host copy of the site list (sorted by emulated rank, local raster)
    std::vector<long long> site_cell;
    std::vector<float> site_thr;
    std::vector<int> site_rank;
    std::unordered_map<long long, size_t> site_index;  // cell -> site, built on demand
    // deck nucleation points: key -> (rank, entry)
    std::vector<std::pair<long long, std::pair<int, int>>> nucpt;
    // orientation injection (host copy): key -> rotmat
    std::vector<long long> inj_key;
    std::vector<double> inj_rot;
    // grain records rebuilt from the device log
    std::vector<mms_grain> grains;
    int grains_synced = 1;
    Ctl *h_ctl = nullptr;  // pinned
    double *h_red = nullptr;  // pinned reduction result
    // h_ctl and h_red as the device addresses them (null: copies instead)
    Ctl *d_hctl = nullptr;
    double *d_hred = nullptr;
    uint64_t launches = 0;
    bool stepped = false;
    std::string err;
    size_t bytes = 0;
    std::vector<void *> allocs;
    void *stage = nullptr;    // field staging buffer for host copies
    size_t stage_bytes = 0;
    int rng_checked_grains = -1;  // grain count at the last orientation-table check
    // z-slab split of one domain: p holds this slab's parameters (its
    // layers of subblocks), gp and gg the whole domain's; ranks holds every
    // emulated rank of the whole domain, of which this slab owns
    // [r0, r0 + ka.g.nranks)
    int nslabs = 1, slab = 0, r0 = 0, kz0 = 0;
    mms_params gp{};
    Geo gg{};
    std::vector<cudaEvent_t> slab_events;  // mms_slab_group_step's ordering events
    // one process per device: the NCCL communicator of the slab group
    // (mms_slab_nccl_init) and 64 bytes of device scratch for its checks
    void *nccl_comm = nullptr;
    void *nccl_scratch = nullptr;
    // XDMF output: rank 0's rand() stream where its first still-undrawn
    // orientation begins (r0_snap_k draws after setup and any renumbering),
    // the grain renumbering of the last write, the time series written
    RngState r0_snap;
    long long r0_snap_k = 0;
    bool r0_snap_valid = false;
    std::vector<uint64_t> renumber;
    std::vector<int64_t> xdmf_series;
    std::string xdmf_base;
    // h_ctl holds the device control block as it stands: set at the end of
    // mms_step, cleared by every call that runs kernels writing the block
    // (steps, the adjoint's record, slab and batch steps, tuning) or writes
    // it from the host; reductions, copies and conversions never write it
    bool ctl_known = false;
    // d.fs_part holds the per-tile fraction-solid sums of the current
    // fields: set by a successful mms_step_reduce whose last stencil left
    // them, cleared by every other step, wherever ctl_known is, and by
    // every call that writes fields or changes the stencil tile
    bool fs_part_valid = false;
    // frozen-CA record for the adjoint
    struct AdjRec {
        unsigned long long t0 = 0;
        long long nrec = 0;
        int every = 0;
        long long nckpt = 0;
        unsigned char *flags = nullptr;  // nrec x N
        double *curv = nullptr;          // nrec x N (TipCurvature)
        char *ckpt = nullptr;            // nckpt x 3 x N x element size
    } adj;
};

namespace {

#define CU(call)                                                                        \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);              \
            return MMS_ERR_CUDA;                                                        \
        }                                                                               \
    } while (0)

template <typename T>
mms_status dalloc(mms_ctx *ctx, T **ptr, size_t count, bool zero = true)
{
    void *p = nullptr;
    size_t bytes = sizeof(T) * (count ? count : 1);
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        ctx->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        return MMS_ERR_NOMEM;
    }
    if (!zero) {
        ctx->allocs.push_back(p);
        ctx->bytes += bytes;
        *ptr = (T *)p;
        return MMS_OK;
    }
    // zeroed before returning: later host copies into this buffer go through
    // the legacy default stream, which does not wait for ctx->stream
    e = cudaMemsetAsync(p, 0, bytes, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(p);
        ctx->err = std::string("cudaMemsetAsync: ") + cudaGetErrorString(e);
        return MMS_ERR_CUDA;
    }
    ctx->allocs.push_back(p);
    ctx->bytes += bytes;
    *ptr = (T *)p;
    return MMS_OK;
}

// A field the stencil reads and writes (ce, cl, fs, gr, the AM
// temperature): allocated with 16 bytes of room in front and placed
// 16 - es bytes past a 16-byte boundary, so that interior cell 1 of every
// row is 16-byte aligned (rows are a multiple of 8 elements).  The stencil
// moves pairs of cells as single words, and its tensor maps start at that
// boundary.
template <typename T>
mms_status dalloc_field(mms_ctx *ctx, T **ptr, size_t count, size_t es = sizeof(T))
{
    char *raw = nullptr;
    mms_status st = dalloc(ctx, &raw, count * es + 16);
    if (st) return st;
    *ptr = (T *)(raw + 16 - es);
    return MMS_OK;
}

// NVTX range over a library call or a phase of one (Nsight Systems and
// other NVTX tools show them; without a tool attached the calls do nothing)
struct Range {
    explicit Range(const char *name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range &) = delete;
    Range &operator=(const Range &) = delete;
};

constexpr int GRAPH_STEPS = 8;

void drop_graph(mms_ctx *ctx)
{
    if (ctx->step_graph) cudaGraphExecDestroy(ctx->step_graph);
    ctx->step_graph = nullptr;
    if (ctx->multi_graph) cudaGraphExecDestroy(ctx->multi_graph);
    ctx->multi_graph = nullptr;
    if (ctx->sum_graph) cudaGraphExecDestroy(ctx->sum_graph);
    ctx->sum_graph = nullptr;
}

void dfree(mms_ctx *ctx, void *p)
{
    if (!p) return;
    cudaFree(p);
    ctx->allocs.erase(std::remove(ctx->allocs.begin(), ctx->allocs.end(), p), ctx->allocs.end());
}

// Host <-> device copies ordered on the context's stream and complete on
// return.  (A plain cudaMemcpy from pageable memory may return before its
// DMA has landed, and it is not ordered with the context's non-blocking
// stream, whose kernels could then read a partly copied buffer.)
cudaError_t h2d(mms_ctx *ctx, void *dst, const void *src, size_t bytes)
{
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
    return e == cudaSuccess ? cudaStreamSynchronize(ctx->stream) : e;
}

cudaError_t d2h(mms_ctx *ctx, void *dst, const void *src, size_t bytes)
{
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    return e == cudaSuccess ? cudaStreamSynchronize(ctx->stream) : e;
}

cudaError_t dzero(mms_ctx *ctx, void *dst, size_t bytes)
{
    cudaError_t e = cudaMemsetAsync(dst, 0, bytes, ctx->stream);
    return e == cudaSuccess ? cudaStreamSynchronize(ctx->stream) : e;
}

// device-layout and reference-layout linear indices (see Geo)
long long cidx(const Geo &g, long long i, long long j, long long k) { return dev_index(g, i, j, k); }
long long rcidx(const Geo &g, long long i, long long j, long long k) { return ref_index(g, i, j, k); }

// Pitched copies between the device layout and a caller's buffer in the
// reference layout (rows of gx+2 elements of es bytes).
cudaError_t copy_out(mms_ctx *ctx, void *host, const void *dev, size_t es);
cudaError_t copy_in(mms_ctx *ctx, void *dev, const void *host, size_t es);

// Extract the sparse site list in (rank, local raster) order from the
// whole domain's threshold array (reference layout), for this context's ranks.
void extract_sites(mms_ctx *ctx, const std::vector<float> &thr)
{
    const mms_params &p = ctx->p;
    const Geo &g = ctx->ka.g;
    ctx->site_cell.clear();
    ctx->site_thr.clear();
    ctx->site_rank.clear();
    ctx->site_index.clear();
    for (int ri = 0; ri < g.nranks; ri++) {
        const Rank &r = ctx->ranks[ctx->r0 + ri];
        for (long long z = 1; z <= p.gsdimz; z++)
            for (long long y = 1; y <= p.gsdimy; y++)
                for (long long x = 1; x <= p.gsdimx; x++) {
                    long long I = (long long)r.sbx * p.gsdimx + x, J = (long long)r.sby * p.gsdimy + y,
                              K = (long long)r.sbz * p.gsdimz + z;
                    long long c = rcidx(ctx->gg, I, J, K);
                    if (thr[c] != INFINITY) {
                        ctx->site_cell.push_back(cidx(g, I, J, K - ctx->kz0));
                        ctx->site_thr.push_back(thr[c]);
                        ctx->site_rank.push_back(ri);
                    }
                }
    }
}

mms_status upload_sites(mms_ctx *ctx)
{
    DevPtrs &d = ctx->ka.d;
    dfree(ctx, d.site_cell);
    dfree(ctx, d.site_thr);
    dfree(ctx, d.site_rank);
    dfree(ctx, d.site_flag);
    dfree(ctx, d.cand);
    dfree(ctx, d.cand_stage);
    dfree(ctx, d.nuc_blk_cnt);
    dfree(ctx, d.cand_ex);
    d.site_cell = nullptr;
    d.site_thr = nullptr;
    d.site_rank = nullptr;
    d.site_flag = nullptr;
    d.cand = nullptr;
    d.cand_stage = nullptr;
    d.nuc_blk_cnt = nullptr;
    d.cand_ex = nullptr;
    drop_graph(ctx);
    size_t n = ctx->site_cell.size();
    d.nsites = (long long)n;
    d.nuc_blocks = (int)std::max<size_t>(1, (n + 255) / 256);
    mms_status st;
    if ((st = dalloc(ctx, &d.site_cell, n)) || (st = dalloc(ctx, &d.site_thr, n)) ||
        (st = dalloc(ctx, &d.site_rank, n)) || (st = dalloc(ctx, &d.site_flag, n)) || (st = dalloc(ctx, &d.cand, n)) ||
        (st = dalloc(ctx, &d.cand_stage, (size_t)d.nuc_blocks * 256)) || (st = dalloc(ctx, &d.nuc_blk_cnt, d.nuc_blocks)) ||
        (st = dalloc(ctx, &d.cand_ex, n)))
        return st;
    if (n) {
        CU(cudaMemcpyAsync(d.site_cell, ctx->site_cell.data(), n * sizeof(long long), cudaMemcpyHostToDevice, ctx->stream));
        CU(cudaMemcpyAsync(d.site_thr, ctx->site_thr.data(), n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        CU(cudaMemcpyAsync(d.site_rank, ctx->site_rank.data(), n * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    }
    CU(cudaStreamSynchronize(ctx->stream));
    return MMS_OK;
}

// nuc_pt lookup table: key = global halo'd cell, first entry of the rank's
// list wins (createGrains' linear search, grain.c:392-401).
mms_status upload_nucpt(mms_ctx *ctx)
{
    const Geo &g = ctx->ka.g;
    DevPtrs &d = ctx->ka.d;
    ctx->nucpt.clear();
    for (int ri = 0; ri < g.nranks; ri++) {
        const int R = ctx->r0 + ri;
        const Rank &r = ctx->ranks[R];
        for (int j = 0; j < (int)r.nuc.size(); j++) {
            const NucPt &n = r.nuc[j];
            const long long kz = (long long)n.cz - ctx->kz0;
            if (n.cx >= (size_t)g.gx || n.cy >= (size_t)g.gy || kz < 0 || kz >= g.gz) continue;
            long long key = cidx(g, (long long)n.cx + 1, (long long)n.cy + 1, kz + 1);
            ctx->nucpt.push_back({key, {R, j}});
        }
    }
    std::stable_sort(ctx->nucpt.begin(), ctx->nucpt.end(),
                     [](const auto &a, const auto &b) { return a.first < b.first; });
    size_t n = ctx->nucpt.size();
    std::vector<long long> keys(n), entry(n);
    std::vector<double> rot(9 * (n ? n : 1));
    for (size_t i = 0; i < n; i++) {
        keys[i] = ctx->nucpt[i].first;
        entry[i] = ((long long)ctx->nucpt[i].second.first << 32) | (unsigned)ctx->nucpt[i].second.second;
        const NucPt &np = ctx->ranks[ctx->nucpt[i].second.first].nuc[ctx->nucpt[i].second.second];
        rotmat_from_angles(np.gx, np.gy, np.gz, &rot[9 * i]);
    }
    mms_status st;
    dfree(ctx, d.nucpt_key);
    dfree(ctx, d.nucpt_entry);
    dfree(ctx, d.nucpt_rot);
    if ((st = dalloc(ctx, &d.nucpt_key, n)) || (st = dalloc(ctx, &d.nucpt_entry, n)) || (st = dalloc(ctx, &d.nucpt_rot, 9 * n)))
        return st;
    d.n_nucpt = (long long)n;
    if (n) {
        CU(cudaMemcpyAsync(d.nucpt_key, keys.data(), n * sizeof(long long), cudaMemcpyHostToDevice, ctx->stream));
        CU(cudaMemcpyAsync(d.nucpt_entry, entry.data(), n * sizeof(long long), cudaMemcpyHostToDevice, ctx->stream));
        CU(cudaMemcpyAsync(d.nucpt_rot, rot.data(), 9 * n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    }
    CU(cudaStreamSynchronize(ctx->stream));
    return MMS_OK;
}

// Refill every rank's device table of orientation draws so that it starts
// at the first unconsumed draw.  Called only with the stream idle.
mms_status refill_rng(mms_ctx *ctx, bool force)
{
    const Geo &g = ctx->ka.g;
    DevPtrs &d = ctx->ka.d;
    if (!ctx->p.gnUseOrientation) return MMS_OK;
    // draws are consumed only by new grains: nothing to check otherwise;
    // no rank past half its table: no refill yet
    if (!force && ctx->h_ctl->num_grains == ctx->rng_checked_grains) return MMS_OK;
    ctx->rng_checked_grains = ctx->h_ctl->num_grains;
    if (!force && (long long)ctx->h_ctl->rng_used_max * 2 <= d.rng_cap) return MMS_OK;
    std::vector<int> used(g.nranks);
    CU(d2h(ctx, used.data(), d.rng_used, sizeof(int) * g.nranks));
    bool any = force;
    for (int r = 0; r < g.nranks; r++)
        if (used[r] * 2 > d.rng_cap) any = true;
    if (!any) return MMS_OK;
    std::vector<double> tab((size_t)g.nranks * d.rng_cap * 9);
    std::vector<long long> base(g.nranks);
    for (int ri = 0; ri < g.nranks; ri++) {
        Rank &r = ctx->ranks[ctx->r0 + ri];
        if (ctx->r0 + ri == 0 && !ctx->r0_snap_valid) {
            // rank 0's stream before its first orientation draw
            r.save(ctx->r0_snap);
            ctx->r0_snap_k = (long long)r.angles.size();
            ctx->r0_snap_valid = true;
        }
        r.rng_base += used[ri];
        while ((long long)r.angles.size() < r.rng_base + d.rng_cap) {
            NucPt n{};
            draw_orientation(ctx->p, r, n);
            r.angles.push_back({n.gx, n.gy, n.gz});
        }
        for (int k = 0; k < d.rng_cap; k++) {
            const auto &a = r.angles[r.rng_base + k];
            rotmat_from_angles(a[0], a[1], a[2], &tab[((size_t)ri * d.rng_cap + k) * 9]);
        }
        base[ri] = r.rng_base;
    }
    CU(h2d(ctx, d.rng_rot, tab.data(), tab.size() * sizeof(double)));
    CU(h2d(ctx, d.rng_base, base.data(), sizeof(long long) * g.nranks));
    CU(dzero(ctx, d.rng_used, sizeof(int) * g.nranks));
    CU(dzero(ctx, &d.ctl->rng_used_max, sizeof(int)));
    ctx->h_ctl->rng_used_max = 0;
    return MMS_OK;
}

void set_status(mms_ctx *ctx, mms_status s, const char *msg)
{
    if (msg) ctx->err = msg;
    (void)s;
}

mms_status read_ctl(mms_ctx *ctx)
{
    CU(cudaMemcpyAsync(ctx->h_ctl, ctx->ka.d.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    if (ctx->prof) ctx->prof->collect();
    return MMS_OK;
}

int launch_one_step(mms_ctx *ctx, int start_stage, bool sumfs = false);

AmParams am_params(const mms_params &p)
{
    AmParams m;
    m.lsd = p.lsd;
    m.lv = p.lv;
    m.lhs = p.lhs;
    m.lab = p.lab;
    m.lpow = p.lpow;
    m.liniT = p.liniT;
    m.lthcon = p.lthcon;
    m.rho_cp = p.rho * p.lcp;
    m.x0 = p.x0;
    m.y0 = p.y0;
    m.z0 = p.z0;
    m.amtracks = p.amtracks;
    m.nsbx_times_sbx = p.gnsbx * p.gsdimx;
    return m;
}

// Captures one whole step, and GRAPH_STEPS consecutive steps, into graphs
// (once per kernel-argument set).  A step that stalls turns the kernels
// after it into no-ops, so a multi-step graph stops where separate
// launches would.
mms_status ensure_graph(mms_ctx *ctx)
{
    if (ctx->step_graph && ctx->multi_graph && ctx->sum_graph) return MMS_OK;
    EventProfiler *saved = ctx->prof;
    ctx->prof = nullptr;
    auto capture = [&](int steps, cudaGraphExec_t *out, bool sumfs = false) -> int {
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return -1;
        int n = 0;
        for (int k = 0; k < steps; k++) n += launch_one_step(ctx, 0, sumfs);
        if (cudaStreamEndCapture(ctx->stream, &g) != cudaSuccess) return -1;
        const cudaError_t e = cudaGraphInstantiate(out, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            *out = nullptr;
            return -1;
        }
        return n;
    };
    const int n1 = ctx->step_graph ? ctx->step_graph_kernels : capture(1, &ctx->step_graph);
    const int nm = n1 >= 0 && !ctx->multi_graph ? capture(GRAPH_STEPS, &ctx->multi_graph) : 0;
    const int ns = n1 >= 0 && nm >= 0 && !ctx->sum_graph ? capture(1, &ctx->sum_graph, true) : 0;
    ctx->prof = saved;
    if (n1 < 0 || nm < 0 || ns < 0) {
        drop_graph(ctx);
        ctx->err = "capturing the step graphs failed";
        return MMS_ERR_CUDA;
    }
    ctx->step_graph_kernels = n1;
    return MMS_OK;
}

// The step graphs captured ahead of the first step (at creation and after a
// tile change), so that the first stepping call does not pay for the
// capture; a failure here leaves them to be captured by that call.
void prepare_graphs(mms_ctx *ctx)
{
    if (ensure_graph(ctx) != MMS_OK) {
        ctx->err.clear();
        cudaGetLastError();
    }
}

int launch_one_step(mms_ctx *ctx, int start_stage, bool sumfs)
{
    int n = 0;
    const mms_params &p = ctx->p;
    if (start_stage == 0 && p.am) {
        n += launch_temp_am(ctx->ka, am_params(p), ctx->prec, ctx->stream, ctx->prof, ctx->am_rows);
    }
    n += launch_step(ctx->ka, ctx->tma, ctx->prec, ctx->stream, start_stage, ctx->prof, sumfs);
    return n;
}

// Pull grain records created since the last sync and rebuild grain_t.
// A grain made by another slab of a split domain carries its whole-domain
// cell and emulated rank; every slab replays every rank's stream, so its
// orientation draw is found here too.
mms_status sync_grains(mms_ctx *ctx)
{
    mms_status st = read_ctl(ctx);
    if (st) return st;
    int ng = ctx->h_ctl->num_grains;
    if (ng <= ctx->grains_synced) return MMS_OK;
    int first = ctx->grains_synced, cnt = ng - first;
    std::vector<GrainLog> log(cnt);
    CU(d2h(ctx, log.data(), ctx->ka.d.grain_log + first, sizeof(GrainLog) * cnt));
    bool need_rot = false;
    for (const GrainLog &lg : log) need_rot |= (lg.kind == 3) || (lg.kind & GL_REMOTE);
    std::vector<double> rows;
    if (need_rot) {
        rows.resize((size_t)cnt * 9);
        CU(d2h(ctx, rows.data(), ctx->ka.d.grain_rot + 9 * (long long)first, sizeof(double) * 9 * cnt));
    }
    if ((int)ctx->grains.size() < ng) ctx->grains.resize(ng);
    const mms_params &p = ctx->p;
    const Geo &g = ctx->ka.g;
    for (int i = 0; i < cnt; i++) {
        const GrainLog &lg = log[i];
        mms_grain &gr = ctx->grains[first + i];
        std::memset(&gr, 0, sizeof gr);
        if (lg.kind == 3) {
            // pre-filled grain (mms_set_grains): no nucleus, rotation from the table
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) gr.rotmat[a][b] = rows[9 * (size_t)i + 3 * a + b];
            continue;
        }
        const bool remote = (lg.kind & GL_REMOTE) != 0;
        const int kind = lg.kind & ~GL_REMOTE;
        long long c = lg.cell, I, J, K;  // whole-domain interior-based cell coordinates
        if (remote) {
            K = c / ctx->gg.rsz;
            J = (c % ctx->gg.rsz) / ctx->gg.rsy;
            I = c % ctx->gg.rsy;
        } else {
            K = c / g.sz + ctx->kz0;
            J = (c % g.sz) / g.sy;
            I = c % g.sy;
        }
        NucPt nuc{};
        if (kind == 0) {
            int rr = (int)(lg.aux >> 32), jj = (int)(lg.aux & 0xffffffff);
            nuc = ctx->ranks[rr].nuc[jj];
        } else {
            nuc.x = cell2real(p, 0, (double)(I - 1));
            nuc.y = cell2real(p, 1, (double)(J - 1));
            nuc.z = cell2real(p, 2, (double)(K - 1));
            nuc.threshold = (double)lg.thr;
            if (kind == 1) {
                Rank &rk = ctx->ranks[lg.rank];
                while ((long long)rk.angles.size() <= lg.aux) {  // another slab's rank
                    NucPt n{};
                    draw_orientation(ctx->p, rk, n);
                    rk.angles.push_back({n.gx, n.gy, n.gz});
                }
                const auto &a = rk.angles[lg.aux];
                nuc.gx = a[0];
                nuc.gy = a[1];
                nuc.gz = a[2];
            }
        }
        double R[9];
        if (remote) {
            std::memcpy(R, &rows[9 * (size_t)i], sizeof R);
        } else {
            rotmat_from_angles(nuc.gx, nuc.gy, nuc.gz, R);
            auto ik = std::lower_bound(ctx->inj_key.begin(), ctx->inj_key.end(), c);
            if (ik != ctx->inj_key.end() && *ik == c)
                std::memcpy(R, &ctx->inj_rot[9 * (ik - ctx->inj_key.begin())], sizeof R);
        }
        gr.nuc_x = nuc.x;
        gr.nuc_y = nuc.y;
        gr.nuc_z = nuc.z;
        gr.nuc_timestep = lg.timestep;
        gr.nuc_threshold = nuc.threshold;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) gr.rotmat[a][b] = R[3 * a + b];
        gr.rotang[0] = nuc.gx;
        gr.rotang[1] = nuc.gy;
        gr.rotang[2] = nuc.gz;
    }
    ctx->grains_synced = ng;
    return MMS_OK;
}

// staging buffer of one whole field in the reference layout: an FP64 field's
// size from creation on, grown (never shrunk) for wider fields (dc); its
// contents are always written before they are read, so it is not cleared
void *stage_buffer(mms_ctx *ctx, size_t bytes)
{
    if (ctx->stage_bytes < bytes) {
        dfree(ctx, ctx->stage);
        ctx->stage = nullptr;
        ctx->stage_bytes = 0;
        char *p = nullptr;
        if (dalloc(ctx, &p, bytes, false) != MMS_OK) return nullptr;
        ctx->stage = p;
        ctx->stage_bytes = bytes;
    }
    return ctx->stage;
}

// Field copies between the device layout and a caller buffer in the
// reference layout: one contiguous host<->device copy of the whole field
// through a staging buffer, re-pitched on the device (row-by-row 2D copies
// of ~2 KB rows run far below the link's bandwidth).
cudaError_t copy_out(mms_ctx *ctx, void *host, const void *dev, size_t es)
{
    const Geo &g = ctx->ka.g;
    const long long rows = (long long)(g.gy + 2) * (g.gz + 2);
    void *st = stage_buffer(ctx, (size_t)g.rN * es);
    cudaError_t e;
    if (!st) {
        e = cudaMemcpy2DAsync(host, (size_t)g.rsy * es, dev, (size_t)g.P * es, (size_t)g.rsy * es, (size_t)rows,
                              cudaMemcpyDeviceToHost, ctx->stream);
    } else {
        launch_repack(st, g.rsy * (long long)es, dev, g.P * (long long)es, (int)(g.rsy * (long long)es), rows,
                      ctx->stream);
        e = cudaMemcpyAsync(host, st, (size_t)g.rN * es, cudaMemcpyDeviceToHost, ctx->stream);
    }
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(ctx->stream);
}

cudaError_t copy_in(mms_ctx *ctx, void *dev, const void *host, size_t es)
{
    const Geo &g = ctx->ka.g;
    const long long rows = (long long)(g.gy + 2) * (g.gz + 2);
    void *st = stage_buffer(ctx, (size_t)g.rN * es);
    cudaError_t e;
    if (!st) {
        e = cudaMemcpy2DAsync(dev, (size_t)g.P * es, host, (size_t)g.rsy * es, (size_t)g.rsy * es, (size_t)rows,
                              cudaMemcpyHostToDevice, ctx->stream);
    } else {
        e = cudaMemcpyAsync(st, host, (size_t)g.rN * es, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess)
            launch_repack(dev, g.P * (long long)es, st, g.rsy * (long long)es, (int)(g.rsy * (long long)es), rows,
                          ctx->stream);
    }
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(ctx->stream);
}

mms_status create_ctx(const mms_params *pin, int nslabs, int slab, mms_ctx **out);

}  // namespace

const mms_params &ctx_params(const mms_ctx *ctx) { return ctx->p; }

// ============================================================= public ABI
extern "C" {

const char *mms_status_string(mms_status s)
{
    switch (s) {
    case MMS_OK: return "ok";
    case MMS_ERR_ARG: return "invalid argument";
    case MMS_ERR_CUDA: return "CUDA error";
    case MMS_ERR_NO_DEVICE: return "no usable CUDA device";
    case MMS_ERR_COURANT: return "Instability by Courant criterion, lower calculation time step";
    case MMS_ERR_NEGATIVE_CE: return "negative ce: instability by Courant criterion";
    case MMS_ERR_GRAIN_OVERFLOW: return "grain id beyond MaxTotGrains";
    case MMS_ERR_DECK: return "input deck error";
    case MMS_ERR_IO: return "file I/O error";
    case MMS_ERR_TIMEOUT: return "device wait timed out";
    case MMS_ERR_STATE: return "call made in the wrong state";
    case MMS_ERR_NOMEM: return "out of memory";
    case MMS_ERR_SCRATCH_LIMIT: return "grid larger than the fixed device scratch (at most 2^30 interior cells)";
    case MMS_ERR_BOUNDS: return "a kernel index outside its buffer (bounds-checked build)";
    case MMS_ERR_SLAB_CAPACITY: return "more nucleation candidates in one step than the slab's row buffer holds";
    }
    return "unknown status";
}

const char *mms_last_error(const mms_ctx *ctx) { return ctx ? ctx->err.c_str() : ""; }

mms_status mms_set_stream(mms_ctx *ctx, void *cuda_stream)
{
    if (!ctx) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->stream = cuda_stream ? (cudaStream_t)cuda_stream : ctx->own_stream;
    return MMS_OK;
}

mms_status mms_set_profiling(mms_ctx *ctx, int on)
{
    if (!ctx) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    CU(cudaStreamSynchronize(ctx->stream));
    if (on && !ctx->prof) ctx->prof = new EventProfiler();
    if (!on && ctx->prof) {
        ctx->prof->collect();
        delete ctx->prof;
        ctx->prof = nullptr;
    }
    return MMS_OK;
}

mms_status mms_set_stencil_tile(mms_ctx *ctx, int cells_per_thread, int zchunk)
{
    if (!ctx || (cells_per_thread != 1 && cells_per_thread != 2) || zchunk < 0 || zchunk > 64) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->tma.cpt = cells_per_thread;
    ctx->tma.zc = zchunk;
    make_tma(ctx->ka, ctx->prec, ctx->tma);
    drop_graph(ctx);
    ctx->fs_part_valid = false;
    if (ctx->nslabs == 1) prepare_graphs(ctx);
    return MMS_OK;
}

mms_status mms_set_am_tile(mms_ctx *ctx, int rows)
{
    if (!ctx || !(rows == 0 || rows == 256 || (rows >= 64 && rows <= 128 && rows % 16 == 0))) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->am_rows = rows;
    drop_graph(ctx);
    if (ctx->nslabs == 1) prepare_graphs(ctx);
    return MMS_OK;
}

mms_status mms_get_am_tile(const mms_ctx *ctx, int *rows)
{
    if (!ctx || !rows) return MMS_ERR_ARG;
    *rows = ctx->am_rows;
    return MMS_OK;
}

mms_status mms_get_stencil_tile(const mms_ctx *ctx, int *cells_per_thread, int *zchunk)
{
    if (!ctx || !cells_per_thread || !zchunk) return MMS_ERR_ARG;
    *cells_per_thread = ctx->tma.ok ? ctx->tma.cpt : 1;
    *zchunk = ctx->tma.zc;
    return MMS_OK;
}

// Stencil tile autotuner.  Every candidate (cells per thread x z-chunk) runs
// the diffusion + fs-change kernel on a shadow of the fields it writes (ce,
// the next cl and fs, gr, the solid bitmask, the control block), so the
// domain's state is untouched; the candidate with the lowest median time
// over `reps` launches is kept.
mms_status mms_autotune(mms_ctx *ctx, int reps, int *cells_per_thread, int *zchunk, double *best_ms)
{
    Range range("mms_autotune");
    if (ctx) ctx->ctl_known = ctx->fs_part_valid = false;
    if (!ctx || reps < 1) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    mms_status rs0 = read_ctl(ctx);
    if (rs0) return rs0;
    const Geo &g = ctx->ka.g;
    const size_t N = (size_t)g.N;
    const size_t rs = ctx->prec == MMS_PREC_F32 ? sizeof(float) : sizeof(double);
    KernelArgs sa = ctx->ka;
    const int pout = (int)((ctx->h_ctl->timestep + 1) & 1ULL);
    std::vector<void *> shadow;
    // es > 0: a field, placed as dalloc_field places it (es = its element size)
    auto shadow_of = [&](const void *src, size_t bytes, void **dst, size_t es = 0) -> cudaError_t {
        void *raw = nullptr;
        cudaError_t e = cudaMalloc(&raw, bytes + (es ? 16 : 0));
        if (e != cudaSuccess) return e;
        shadow.push_back(raw);
        *dst = es ? (void *)((char *)raw + 16 - es) : raw;
        return cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyDeviceToDevice, ctx->stream);
    };
    auto release = [&]() {
        cudaStreamSynchronize(ctx->stream);
        for (void *q : shadow) cudaFree(q);
    };
    void *sce, *scl, *sfs, *sgr, *sbits, *sctl;
    cudaError_t e;
    if ((e = shadow_of(sa.d.ce, N * rs, &sce, rs)) || (e = shadow_of(sa.d.cl[pout], N * rs, &scl, rs)) ||
        (e = shadow_of(sa.d.fs[pout], N * rs, &sfs, rs)) || (e = shadow_of(sa.d.gr, N * sizeof(int), &sgr, 4)) ||
        (e = shadow_of(sa.d.solid_bits, (size_t)g.nwords * sizeof(unsigned), &sbits)) ||
        (e = shadow_of(sa.d.ctl, sizeof(Ctl), &sctl))) {
        release();
        ctx->err = std::string("autotune shadow buffers: ") + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? MMS_ERR_NOMEM : MMS_ERR_CUDA;
    }
    sa.d.ce = sce;
    sa.d.cl[pout] = scl;
    sa.d.fs[pout] = sfs;
    sa.d.gr = (int *)sgr;
    sa.d.solid_bits = (unsigned *)sbits;
    sa.d.ctl = (Ctl *)sctl;
    Ctl c = *ctx->h_ctl;
    c.timestep += 1;
    c.status = 0;
    c.stall = 0;
    cudaMemcpyAsync(sctl, &c, sizeof c, cudaMemcpyHostToDevice, ctx->stream);

    struct Cand {
        int cpt, zc;
    };
    std::vector<Cand> cands;
    for (int cpt = 1; cpt <= (ctx->tma.ok ? 2 : 1); cpt++)
        for (int zc : {0, 8, 16, 32})
            if (zc <= g.gz) cands.push_back({cpt, zc});
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 1e300;
    Cand pick{ctx->tma.cpt, ctx->tma.zc};
    // the candidates' launches interleaved round by round, so that a drift
    // of the clocks during the tuning weighs on every candidate alike
    std::vector<TmaHolder> ths;
    std::vector<Cand> live;
    for (const Cand &cd : cands) {
        TmaHolder th{};
        th.cpt = cd.cpt;
        th.zc = cd.zc;
        if (ctx->tma.ok && !make_tma(sa, ctx->prec, th)) continue;
        ths.push_back(th);
        live.push_back(cd);
    }
    std::vector<std::vector<float>> ms(live.size());
    for (int r = 0; r < reps + 2; r++)
        for (size_t c = 0; c < live.size(); c++) {
            cudaEventRecord(e0, ctx->stream);
            launch_stencil(sa, ths[c], ctx->prec, ctx->stream);
            cudaEventRecord(e1, ctx->stream);
            cudaEventSynchronize(e1);
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            if (r >= 2) ms[c].push_back(t);
        }
    if ((e = cudaGetLastError()) != cudaSuccess) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        release();
        ctx->err = std::string("autotune launch: ") + cudaGetErrorString(e);
        return MMS_ERR_CUDA;
    }
    for (size_t c = 0; c < live.size(); c++) {
        std::sort(ms[c].begin(), ms[c].end());
        const double med = ms[c][ms[c].size() / 2];
        if (med < best) {
            best = med;
            pick = live[c];
        }
    }
    // FP32 AM form: the contraction's tile (128-row tiles with two
    // accumulator sets, or 256-row tiles with one), timed with the tables on
    // shadows of the temperature and the layer flag; the tables are scratch
    // rebuilt by every step, and are rebuilt for the current step afterwards
    int am_rows = ctx->am_rows;
    if (ctx->ka.p.temp_mode == 2 && ctx->prec == MMS_PREC_F32) {
        void *sT = nullptr, *sls = nullptr;
        if ((e = shadow_of(sa.d.T32, N * sizeof(float), &sT, 4)) ||
            (sa.d.lsindex && (e = shadow_of(sa.d.lsindex, N * sizeof(int), &sls)))) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            release();
            ctx->err = std::string("autotune shadow buffers: ") + cudaGetErrorString(e);
            return e == cudaErrorMemoryAllocation ? MMS_ERR_NOMEM : MMS_ERR_CUDA;
        }
        sa.d.T32 = (float *)sT;
        if (sls) sa.d.lsindex = (int *)sls;
        const AmParams m = am_params(ctx->p);
        double best_am = 1e300;
        const int am_cands[2] = {128, 256};
        std::vector<float> am_ms[2];
        for (int r = 0; r < reps + 2; r++)
            for (int ci = 0; ci < 2; ci++) {
                cudaEventRecord(e0, ctx->stream);
                launch_temp_am(sa, m, ctx->prec, ctx->stream, nullptr, am_cands[ci]);
                cudaEventRecord(e1, ctx->stream);
                cudaEventSynchronize(e1);
                float t = 0.f;
                cudaEventElapsedTime(&t, e0, e1);
                if (r >= 2) am_ms[ci].push_back(t);
            }
        for (int ci = 0; ci < 2; ci++) {
            std::sort(am_ms[ci].begin(), am_ms[ci].end());
            if (am_ms[ci][am_ms[ci].size() / 2] < best_am) {
                best_am = am_ms[ci][am_ms[ci].size() / 2];
                am_rows = am_cands[ci];
            }
        }
        Ctl c2 = c;
        c2.timestep = ctx->h_ctl->timestep >= 1 ? ctx->h_ctl->timestep - 1 : 0;
        cudaMemcpyAsync(sctl, &c2, sizeof c2, cudaMemcpyHostToDevice, ctx->stream);
        launch_temp_am(sa, m, ctx->prec, ctx->stream, nullptr, am_rows);
        if ((e = cudaGetLastError()) != cudaSuccess) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            release();
            ctx->err = std::string("autotune launch: ") + cudaGetErrorString(e);
            return MMS_ERR_CUDA;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    release();
    ctx->tma.cpt = pick.cpt;
    ctx->tma.zc = pick.zc;
    ctx->am_rows = am_rows;
    make_tma(ctx->ka, ctx->prec, ctx->tma);
    drop_graph(ctx);
    if (ctx->nslabs == 1) prepare_graphs(ctx);
    if (cells_per_thread) *cells_per_thread = pick.cpt;
    if (zchunk) *zchunk = pick.zc;
    if (best_ms) *best_ms = best;
    return MMS_OK;
}

int mms_kernel_count(void) { return mms::KID_COUNT; }

const char *mms_kernel_name(int id)
{
    static const char *names[mms::KID_COUNT] = {"k_temp_am", "k_nuc", "k_act", "k_curv", "k_diffuse_fs", "k_list", "k_capture"};
    return (id >= 0 && id < mms::KID_COUNT) ? names[id] : "";
}

mms_status mms_kernel_stats(mms_ctx *ctx, int id, double *total_ms, uint64_t *launches)
{
    if (!ctx || id < 0 || id >= mms::KID_COUNT || !total_ms || !launches) return MMS_ERR_ARG;
    if (!ctx->prof) {
        *total_ms = 0;
        *launches = 0;
        return MMS_OK;
    }
    cudaSetDevice(ctx->device);
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->prof->collect();
    *total_ms = ctx->prof->total_ms[id];
    *launches = ctx->prof->count[id];
    return MMS_OK;
}
uint64_t mms_kernel_launches(const mms_ctx *ctx) { return ctx ? ctx->launches : 0; }
size_t mms_num_cells(const mms_ctx *ctx) { return ctx ? (size_t)ctx->ka.g.rN : 0; }
int mms_uses_tma(const mms_ctx *ctx) { return ctx ? ctx->tma.ok : 0; }

mms_status mms_create(const mms_params *pin, mms_ctx **out) { return create_ctx(pin, 1, 0, out); }

mms_status mms_slab_create(const mms_params *global, int nslabs, int slab, mms_ctx **out)
{
    return create_ctx(global, nslabs, slab, out);
}

}  // extern "C"

namespace {

// Layers of subblocks [L0, L1) of slab `slab` of nslabs (as even as integer
// division makes them).
bool slab_span(const mms_params &p, int nslabs, int slab, int &L0, int &L1)
{
    if (nslabs < 1 || slab < 0 || slab >= nslabs || nslabs > p.gnsbz) return false;
    L0 = (int)((long long)slab * p.gnsbz / nslabs);
    L1 = (int)((long long)(slab + 1) * p.gnsbz / nslabs);
    return true;
}

// Largest number of nucleation sites any slab holds: the capacity of every
// slab's row buffer of new grains (the same on every slab, computed from
// the whole domain's thresholds).
int slab_capacity(const mms_ctx *ctx, const std::vector<float> &thr)
{
    const Geo &G = ctx->gg;
    std::vector<long long> per_plane((size_t)G.gz + 2, 0);
    for (long long K = 1; K <= G.gz; K++)
        for (long long J = 1; J <= G.gy; J++)
            for (long long I = 1; I <= G.gx; I++)
                if (thr[(size_t)rcidx(G, I, J, K)] != INFINITY) per_plane[K]++;
    long long cap = 1;
    for (int s = 0; s < ctx->nslabs; s++) {
        int L0, L1;
        slab_span(ctx->gp, ctx->nslabs, s, L0, L1);
        long long n = 0;
        for (long long K = (long long)L0 * G.sbz + 1; K <= (long long)L1 * G.sbz; K++) n += per_plane[K];
        cap = std::max(cap, n);
    }
    return (int)std::min<long long>(cap, 1LL << 30);
}

// mms_params.site_setup 1: the volume and surface sites of
// init_sb_nucleation (grain.c:930-1010) drawn on the device (sites.cu), with
// each rank's selection probability the reference's site count over its
// candidate cells: floor(rho_v V dx^3) / V and floor(rho_s S dx^2) / S, V
// its non-mold cells (all interior cells) and S those next to a pad face;
// the deck-defined sites of the ranks are presets, the last one at a cell
// winning, as the dense writes of init_sb_nucleation leave them.
mms_status device_sites(mms_ctx *ctx)
{
    const mms_params &P = ctx->gp;
    const Geo &G = ctx->gg, &g = ctx->ka.g;
    const int nr = G.nranks;
    const long long sbc = G.sbcells;
    std::vector<double> pv((size_t)nr), ps((size_t)nr);
    // indices of [lo, hi] (1-based, whole domain of n) not on a pad face
    auto inner = [](long long lo, long long hi, long long n, int pad) {
        long long c = hi - lo + 1;
        if (pad) {
            if (lo <= 1 && 1 <= hi) c--;
            if (n != 1 && lo <= n && n <= hi) c--;
        }
        return c;
    };
    std::map<long long, float> pre;
    for (int r = 0; r < nr; r++) {
        Rank &rk = ctx->ranks[r];
        rk.ncalls_presb = rk.ncalls;
        const long long v = sbc;
        const long long nin = inner((long long)rk.sbx * P.gsdimx + 1, (long long)(rk.sbx + 1) * P.gsdimx, G.gx, P.padBndyX) *
                              inner((long long)rk.sby * P.gsdimy + 1, (long long)(rk.sby + 1) * P.gsdimy, G.gy, P.padBndyY) *
                              inner((long long)rk.sbz * P.gsdimz + 1, (long long)(rk.sbz + 1) * P.gsdimz, G.gz, P.padBndyZ);
        const long long sn = v - nin;
        size_t cv = (size_t)(P.maxGrainDensity * (v * pow(P.cellSize, 3.0)));
        cv = std::min<size_t>(cv, (size_t)v);
        pv[r] = v ? (double)cv / (double)v : 0.0;
        size_t cs = 0;
        if (P.doSurfaceNuc && (P.maxGrainDensitySurf > 0.0)) cs = (size_t)(P.maxGrainDensitySurf * (sn * pow(P.cellSize, 2.0)));
        cs = std::min<size_t>(cs, (size_t)sn);
        ps[r] = sn ? (double)cs / (double)sn : 0.0;
        for (const NucPt &n : rk.nuc) {
            const long long lx = (long long)(n.cx % (size_t)P.gsdimx), ly = (long long)(n.cy % (size_t)P.gsdimy),
                            lz = (long long)(n.cz % (size_t)P.gsdimz);
            pre[(long long)r * sbc + (lz * P.gsdimy + ly) * P.gsdimx + lx] = (float)n.threshold;
        }
    }
    std::vector<long long> pq;
    std::vector<float> pt;
    for (const auto &kv : pre) {
        pq.push_back(kv.first);
        pt.push_back(kv.second);
    }
    SiteDrawArgs a{};
    a.total = (long long)g.nranks * sbc;
    a.qbase = (long long)ctx->r0 * sbc;
    a.sbcells = sbc;
    a.sbx = P.gsdimx;
    a.sby = P.gsdimy;
    a.sbz = P.gsdimz;
    a.nsbx = P.gnsbx;
    a.nsby = P.gnsby;
    a.gx = G.gx;
    a.gy = G.gy;
    a.gz = G.gz;
    a.padx = P.padBndyX;
    a.pady = P.padBndyY;
    a.padz = P.padBndyZ;
    a.rank0 = ctx->r0;
    a.kz0 = ctx->kz0;
    a.dsy = g.sy;
    a.dsz = g.sz;
    a.seed = P.base_random_seed;
    a.vol_centre = P.gnGaussCenter;
    a.vol_sigma = P.gnGaussSigma;
    a.surf_centre = P.gnGaussCenterSurf;
    a.surf_sigma = P.gnGaussSigmaSurf;
    ctx->site_index.clear();
    if (site_draw_device(a, pv, ps, pq, pt, ctx->site_cell, ctx->site_thr, ctx->site_rank, ctx->err))
        return MMS_ERR_CUDA;
    return MMS_OK;
}

mms_status alloc_slab_rows(mms_ctx *ctx, int cap)
{
    DevPtrs &d = ctx->ka.d;
    if (ctx->nslabs < 2) return MMS_OK;
    if (d.x2_send && d.slab_cap == cap) return MMS_OK;
    dfree(ctx, d.x2_send);
    dfree(ctx, d.x2_recv);
    d.x2_send = d.x2_recv = nullptr;
    d.slab_cap = cap;
    drop_graph(ctx);
    mms_status st;
    if ((st = dalloc(ctx, &d.x2_send, (size_t)cap)) || (st = dalloc(ctx, &d.x2_recv, (size_t)cap * ctx->nslabs)))
        return st;
    return MMS_OK;
}

mms_status create_ctx(const mms_params *pin, int nslabs, int slab, mms_ctx **out)
{
    if (!pin || !out) return MMS_ERR_ARG;
    *out = nullptr;
    const mms_params &p0 = *pin;
    int L0 = 0, L1 = 0;
    if (p0.gnsbz < 1 || !slab_span(p0, nslabs, slab, L0, L1)) return MMS_ERR_ARG;
    // the curvature stencil reaches three planes, beyond a slab's one-plane halo
    if (nslabs > 1 && p0.tip_curv) return MMS_ERR_ARG;
    if (p0.site_setup != 0 && p0.site_setup != 1) return MMS_ERR_ARG;
    // device-drawn sites give no whole-domain site count for the slabs' row buffers
    if (nslabs > 1 && p0.site_setup) return MMS_ERR_ARG;
    if (p0.gnsbx < 1 || p0.gnsby < 1 || p0.gnsbz < 1 || p0.gsdimx < 1 || p0.gsdimy < 1 || p0.gsdimz < 1 ||
        p0.cellSize <= 0 || p0.ts_delt <= 0 || p0.maxTotalGrains < 1 || p0.maxTotalGrains > 0x7ffffffeULL)
        return MMS_ERR_ARG;
    if ((!p0.padBndyX && p0.gnsbx > 1) || (!p0.padBndyY && p0.gnsby > 1) || (!p0.padBndyZ && p0.gnsbz > 1))
        return MMS_ERR_ARG;  // periodic exchange between subblocks is not supported
    if (p0.am && p0.thermal_ana != 1) return MMS_ERR_ARG;
    if (p0.precision != MMS_PREC_F64 && p0.precision != MMS_PREC_F32) return MMS_ERR_ARG;
    // Courant check, growth.c:38-50
    double dtx = p0.ts_delt / (p0.cellSize * p0.cellSize);
    if (p0.Dsol * dtx > p0.courant_limit || p0.Dliq * dtx > p0.courant_limit) return MMS_ERR_COURANT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= p0.device) return MMS_ERR_NO_DEVICE;

    mms_ctx *ctx = new mms_ctx();
    ctx->p = p0;
    for (int i = 0; i < p0.n_fixed_nucs; i++) ctx->fixed.push_back(p0.fixed_nucs[i]);
    for (int i = 0; i < p0.n_nuc_volumes; i++) ctx->vols.push_back(p0.nuc_volumes[i]);
    ctx->p.fixed_nucs = nullptr;
    ctx->p.nuc_volumes = nullptr;
    ctx->gp = ctx->p;
    ctx->nslabs = nslabs;
    ctx->slab = slab;
    ctx->p.gnsbz = L1 - L0;
    ctx->kz0 = L0 * p0.gsdimz;
    ctx->r0 = L0 * p0.gnsbx * p0.gnsby;
    ctx->prec = p0.precision;
    ctx->device = p0.device;
    const mms_params &p = ctx->p;
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        delete ctx;
        return MMS_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, ctx->device);
    if (prop.major < 10) {
        delete ctx;
        return MMS_ERR_NO_DEVICE;
    }
    cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
    ctx->stream = ctx->own_stream;
    cudaMallocHost((void **)&ctx->h_ctl, sizeof(Ctl));
    cudaMallocHost((void **)&ctx->h_red, sizeof(double));
    if (!ctx->h_ctl || !ctx->h_red || cudaHostGetDevicePointer((void **)&ctx->d_hctl, ctx->h_ctl, 0) != cudaSuccess ||
        cudaHostGetDevicePointer((void **)&ctx->d_hred, ctx->h_red, 0) != cudaSuccess) {
        ctx->d_hctl = nullptr;
        ctx->d_hred = nullptr;
        cudaGetLastError();
    }

    ctx->gg = make_geo(ctx->gp);
    ctx->ka.g = make_geo(p);
    Geo &g = ctx->ka.g;
    // a slab's inner z faces border the neighbouring slab, not the mold
    g.padz_lo = (slab == 0) ? p0.padBndyZ : 0;
    g.padz_hi = (slab == nslabs - 1) ? p0.padBndyZ : 0;

    Phys &ph = ctx->ka.p;
    ph.rs = p.Dsol * dtx;
    ph.rl = p.Dliq * dtx;
    ph.liq_slope = p.m_solute0;
    ph.k_inv = 1.0 / p.part_coef;
    ph.km = 1.0 - p.part_coef;
    ph.km_inv = 1.0 / ph.km;
    ph.m_inv = 1.0 / ph.liq_slope;
    ph.D_xt = (p.Dliq / p.cellSize / p.cellSize) * p.ts_delt;
    ph.cinit = p.Cinit;
    ph.Tliq = p.liquidusTemp;
    ph.Tsol = p.solidusTemp;
    ph.tip_curv = p.tip_curv;
    ph.curv_fixed = p.curvature_corrected;
    ph.gibbs = p.gibbs_coef;
    ph.fsgrow = p.rev_fsgrow;
    ph.max_grains = p.maxTotalGrains;
    ph.ma = p.m_solute0_a;
    ph.mb = p.m_solute0_b;
    ph.mc = p.m_solute0_c;
    ph.temp_mode = (p.thermal_ana == 0 && p.gradient == 0) ? 0 : (!p.am ? 1 : 2);
    ph.T0 = p.initialTemperature;
    ph.cool_rate = p.cool_rate;
    ph.gradient = p.gradient;
    ph.grad_coef = p.grad_coef;
    ph.velocity = p.velocity;
    ph.velo_coef = p.velo_coef;
    ph.ts_delt = p.ts_delt;
    ph.cellSize = p.cellSize;
    for (int a = 0; a < 3; a++) ph.origin[a] = p.origin_offset[a];
    ph.gz_is_one = (ctx->gg.gz == 1);
    ph.kz0 = ctx->kz0;
    ph.am = p.am;
    ph.amlayer = p.amlayer;
    ph.use_orientation = p.gnUseOrientation;
    ph.cellSize3 = pow(p.cellSize, 3.0);

    mms_status st = MMS_OK;
    DevPtrs &d = ctx->ka.d;
    const size_t N = (size_t)g.N;
    const size_t rs = ctx->prec == MMS_PREC_F32 ? sizeof(float) : sizeof(double);
    auto fail = [&](mms_status s) {
        mms_destroy(ctx);
        return s;
    };
    char *tmp;
    if ((st = dalloc_field(ctx, &tmp, N, rs))) return fail(st);
    d.ce = tmp;
    for (int b = 0; b < 2; b++) {
        if ((st = dalloc_field(ctx, &tmp, N, rs))) return fail(st);
        d.cl[b] = tmp;
        if ((st = dalloc_field(ctx, &tmp, N, rs))) return fail(st);
        d.fs[b] = tmp;
    }
    if ((st = dalloc_field(ctx, &d.gr, N)) || (st = dalloc(ctx, &d.dc, N)) || (st = dalloc(ctx, &d.ctl, 1)) ||
        (st = dalloc(ctx, &d.solid_bits, (size_t)g.nwords)))
        return fail(st);
    if (p.am) {
        // the FP32 form keeps the temperature in FP32
        if ((st = (ctx->prec == MMS_PREC_F32 ? dalloc_field(ctx, &d.T32, N) : dalloc_field(ctx, &d.T, N))))
            return fail(st);
        if ((st = dalloc(ctx, &d.am_tab, (size_t)400 * (g.gx + g.gy + g.gz + 6) + (size_t)(g.gz + 2)))) return fail(st);
        if (ctx->prec == MMS_PREC_F32 && (st = dalloc(ctx, &d.am_ximg, (size_t)am_ximg_size(g.gx, g.gy, g.gz)))) return fail(st);
        if (p.amlayer > 1 && (st = dalloc(ctx, &d.lsindex, N))) return fail(st);
    }
    if (p.tip_curv && (st = dalloc(ctx, &d.curv, N))) return fail(st);
    const size_t nb = (size_t)(g.blocks_per_rank * g.nranks);
    if ((st = dalloc(ctx, &d.list_status, nb)) || (st = dalloc(ctx, &d.blk_off, nb)) ||
        (st = dalloc(ctx, &d.rank_gindex, g.nranks)) || (st = dalloc(ctx, &d.rank_dcsize, g.nranks)) ||
        (st = dalloc(ctx, &d.rank_zero_upto, g.nranks)) || (st = dalloc(ctx, &d.rank_dcbase, g.nranks)) ||
        (st = dalloc(ctx, &d.list_cell, (size_t)g.nranks * g.sbcells)) ||
        (st = dalloc(ctx, &d.list_gid, (size_t)g.nranks * g.sbcells)) ||
        (st = dalloc(ctx, &d.dc_tmp, (size_t)g.nranks * (g.sbcells + 101))) ||
        (st = dalloc(ctx, &d.red, 2 * RED_BLOCKS + 1)) || (st = dalloc(ctx, &d.fs_part, 2 * stencil_parts_max(g) + 1)) ||
        (st = dalloc(ctx, &d.act_scratch, 4 * g.nranks)) ||
        (st = dalloc(ctx, &d.rng_used, g.nranks)) || (st = dalloc(ctx, &d.rng_base, g.nranks)) ||
        (st = dalloc(ctx, &d.grain_rot, 9 * (p.maxTotalGrains + 1))) ||
        (st = dalloc(ctx, &d.grain_log, p.maxTotalGrains + 2)))
        return fail(st);
    {
        std::vector<long long> base(g.nranks);
        for (int r = 0; r < g.nranks; r++) base[r] = (long long)r * (g.sbcells + 101);
        if (h2d(ctx, d.rank_dcbase, base.data(), sizeof(long long) * g.nranks) != cudaSuccess)
            return fail(MMS_ERR_CUDA);
    }
    {
        double zr[9];
        rotmat_from_angles(0.0, 0.0, 0.0, zr);
        std::memcpy(d.zero_rot, zr, sizeof zr);
    }

    // every rank of the whole domain and its stream (a slab replays all of
    // them: rank 0 draws sites for every rank, and grain records of other
    // slabs refer to their ranks' draws)
    ctx->ranks.resize(ctx->gg.nranks);
    for (int r = 0; r < ctx->gg.nranks; r++) {
        Rank &rk = ctx->ranks[r];
        rk.sbx = r % p.gnsbx;
        rk.sby = (r / p.gnsbx) % p.gnsby;
        rk.sbz = r / (p.gnsbx * p.gnsby);
        rk.seed_with((unsigned)r + 1 + p.base_random_seed);
    }
    // initial fields: ce = cl = Cinit everywhere, fs = gr = dc = 0 (setup.c:59-79)
    {
        std::vector<double> init(N, p.Cinit);
        double *dtmp;
        if ((st = dalloc(ctx, &dtmp, N))) return fail(st);
        if (h2d(ctx, dtmp, init.data(), N * sizeof(double)) != cudaSuccess)
            return fail(MMS_ERR_CUDA);
        ctx->launches += launch_convert(ctx->ka, ctx->prec, MMS_FIELD_CE, 1, dtmp, ctx->stream);
        ctx->launches += launch_convert(ctx->ka, ctx->prec, MMS_FIELD_CL, 1, dtmp, ctx->stream);
        cudaStreamSynchronize(ctx->stream);
        dfree(ctx, dtmp);
    }
    if (p.am && ctx->prec == MMS_PREC_F32) am_tc_prepare();
    if (p.am && p.amlayer > 1) {
        // tempPrepareSB_int lsindex (temperature.c:183-189) at timestep 0
        ctx->launches += launch_temp_am(ctx->ka, am_params(p), ctx->prec, ctx->stream, nullptr, ctx->am_rows);
    }
    std::vector<float> thr;  // whole domain, reference layout (host site setup)
    if (p.site_setup == 1) {
        assign_deck_sites(ctx->gp, ctx->gg, ctx->fixed, ctx->vols, ctx->ranks);
        if ((st = device_sites(ctx))) return fail(st);
    } else {
        const std::vector<signed char> mold = make_mold(ctx->gg);
        thr.assign((size_t)ctx->gg.rN, INFINITY);
        setup_sites(ctx->gp, ctx->gg, ctx->fixed, ctx->vols, ctx->ranks, thr, mold);
        extract_sites(ctx, thr);
    }
    if ((st = upload_sites(ctx)) || (st = upload_nucpt(ctx))) return fail(st);
    d.nslabs = nslabs;
    d.slab = slab;
    d.rank0 = ctx->r0;
    if (nslabs > 1) {
        if ((st = dalloc(ctx, &d.x1_send, 2)) || (st = dalloc(ctx, &d.x1_recv, 2 * (size_t)nslabs)) ||
            (st = alloc_slab_rows(ctx, slab_capacity(ctx, thr))))
            return fail(st);
    }
    make_tma(ctx->ka, ctx->prec, ctx->tma);
    // orientation tables
    if (p.gnUseOrientation) {
        long long maxsites = 0;
        std::vector<long long> per(g.nranks, 0);
        for (int r : ctx->site_rank) per[r]++;
        for (long long v : per) maxsites = std::max(maxsites, v);
        d.rng_cap = (int)std::min<long long>(std::max<long long>(256, 2 * maxsites + 256), 1 << 22);
        if ((st = dalloc(ctx, &d.rng_rot, (size_t)g.nranks * d.rng_cap * 9))) return fail(st);
        if ((st = refill_rng(ctx, true))) return fail(st);
    }
    {
        Ctl c{};
        c.timestep = 0;
        c.num_grains = 1;  // the "zero" grain (read_ctrl.c:51)
        if (h2d(ctx, d.ctl, &c, sizeof c) != cudaSuccess) return fail(MMS_ERR_CUDA);
    }
    ctx->grains.resize(1);
    std::memset(&ctx->grains[0], 0, sizeof(mms_grain));
    // the host-copy staging buffer for FP64 fields, so the first uploads
    // and downloads do not allocate
    if (!stage_buffer(ctx, (size_t)g.rN * sizeof(double))) return fail(MMS_ERR_NOMEM);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return fail(MMS_ERR_CUDA);
    if (cudaGetLastError() != cudaSuccess) return fail(MMS_ERR_CUDA);
    if (nslabs == 1) prepare_graphs(ctx);
    *out = ctx;
    return MMS_OK;
}

}  // namespace

// ---- NCCL, loaded at run time -------------------------------------------
// The library does not link NCCL: the slab group's exchanges use the entry
// points of the libnccl the caller names (by default "libnccl.so.2", which
// finds a copy already loaded in the process, such as torch's).
struct NcclApi {
    ncclResult_t (*GetUniqueId)(ncclUniqueId *);
    ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int);
    ncclResult_t (*CommDestroy)(ncclComm_t);
    ncclResult_t (*Send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
    ncclResult_t (*Recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
    ncclResult_t (*AllGather)(const void *, void *, size_t, ncclDataType_t, ncclComm_t, cudaStream_t);
    ncclResult_t (*AllReduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                              cudaStream_t);
    ncclResult_t (*GroupStart)();
    ncclResult_t (*GroupEnd)();
    const char *(*GetErrorString)(ncclResult_t);
};

static std::mutex g_nccl_mu;
static NcclApi g_nccl;
static bool g_nccl_ok = false;

static const NcclApi *nccl_api(const char *path, std::string *err)
{
    std::lock_guard<std::mutex> lock(g_nccl_mu);
    if (g_nccl_ok) return &g_nccl;
    void *h = dlopen(path && *path ? path : "libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
    if (!h) {
        if (err) *err = std::string("dlopen NCCL: ") + dlerror();
        return nullptr;
    }
    NcclApi a{};
    bool ok = true;
    auto sym = [&](auto &fn, const char *name) {
        fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
        ok = ok && fn;
    };
    sym(a.GetUniqueId, "ncclGetUniqueId");
    sym(a.CommInitRank, "ncclCommInitRank");
    sym(a.CommDestroy, "ncclCommDestroy");
    sym(a.Send, "ncclSend");
    sym(a.Recv, "ncclRecv");
    sym(a.AllGather, "ncclAllGather");
    sym(a.AllReduce, "ncclAllReduce");
    sym(a.GroupStart, "ncclGroupStart");
    sym(a.GroupEnd, "ncclGroupEnd");
    sym(a.GetErrorString, "ncclGetErrorString");
    if (!ok) {
        if (err) *err = "NCCL library lacks an entry point";
        return nullptr;
    }
    g_nccl = a;
    g_nccl_ok = true;
    return &g_nccl;
}

static void nccl_release(mms_ctx *ctx)
{
    if (ctx->nccl_comm && g_nccl_ok) g_nccl.CommDestroy((ncclComm_t)ctx->nccl_comm);
    ctx->nccl_comm = nullptr;
}

extern "C" {

mms_status mms_destroy(mms_ctx *ctx)
{
    if (!ctx) return MMS_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (void *p : ctx->allocs) cudaFree(p);
    ctx->allocs.clear();
    for (cudaEvent_t e : ctx->slab_events) cudaEventDestroy(e);
    ctx->slab_events.clear();
    nccl_release(ctx);
    if (ctx->h_ctl) cudaFreeHost(ctx->h_ctl);
    if (ctx->h_red) cudaFreeHost(ctx->h_red);
    drop_graph(ctx);
    delete ctx->prof;
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return MMS_OK;
}

mms_status mms_test_hold_list_block(mms_ctx *ctx, int block, unsigned polls)
{
    if (!ctx || block < -1) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    mms_status st = read_ctl(ctx);
    if (st) return st;
    Ctl c = *ctx->h_ctl;
    c.hold_list_block = block + 1;
    c.wait_polls = polls;
    CU(h2d(ctx, ctx->ka.d.ctl, &c, sizeof c));
    *ctx->h_ctl = c;
    return MMS_OK;
}

mms_status mms_set_grains(mms_ctx *ctx, int n, const double *rotmat9)
{
    if (!ctx || n < 0 || (n && !rotmat9)) return MMS_ERR_ARG;
    if (ctx->stepped) return MMS_ERR_STATE;
    ctx->ctl_known = ctx->fs_part_valid = false;
    if ((uint64_t)n + 1 > ctx->p.maxTotalGrains + 1) return MMS_ERR_GRAIN_OVERFLOW;
    cudaSetDevice(ctx->device);
    mms_status st = read_ctl(ctx);
    if (st) return st;
    if (n) {
        CU(h2d(ctx, ctx->ka.d.grain_rot + 9, rotmat9, sizeof(double) * 9 * (size_t)n));
        std::vector<GrainLog> log((size_t)n);
        for (int g = 0; g < n; g++) log[g] = GrainLog{-1, 0ULL, 3, 0, (long long)(g + 1), 0.f, 0};
        CU(h2d(ctx, ctx->ka.d.grain_log + 1, log.data(), sizeof(GrainLog) * (size_t)n));
    }
    Ctl c = *ctx->h_ctl;
    c.num_grains = n + 1;
    CU(h2d(ctx, ctx->ka.d.ctl, &c, sizeof c));
    *ctx->h_ctl = c;
    ctx->grains.assign((size_t)n + 1, mms_grain{});
    for (int g = 0; g < n; g++)
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) ctx->grains[g + 1].rotmat[i][j] = rotmat9[9 * g + 3 * i + j];
    ctx->grains_synced = n + 1;
    return MMS_OK;
}

mms_status mms_set_sites(mms_ctx *ctx, int64_t n, const int32_t *gxyz, const float *thresholds)
{
    if (!ctx || (n && (!gxyz || !thresholds))) return MMS_ERR_ARG;
    if (ctx->stepped) return MMS_ERR_STATE;
    cudaSetDevice(ctx->device);
    const Geo &g = ctx->ka.g, &G = ctx->gg;
    std::vector<float> thr((size_t)G.rN, INFINITY);  // whole domain
    for (int64_t s = 0; s < n; s++) {
        long long x = gxyz[3 * s], y = gxyz[3 * s + 1], z = gxyz[3 * s + 2];
        if (x < 0 || y < 0 || z < 0 || x >= G.gx || y >= G.gy || z >= G.gz) return MMS_ERR_ARG;
        thr[rcidx(G, x + 1, y + 1, z + 1)] = thresholds[s];
    }
    // rewind every stream to where init_sb_nucleation would start drawing
    for (Rank &r : ctx->ranks) {
        long keep = r.ncalls_presb;
        r.seed_with(r.seed);
        while (r.ncalls < keep) r.rand_();
        r.angles.clear();
        r.rng_base = 0;
    }
    ctx->r0_snap_valid = false;
    extract_sites(ctx, thr);
    mms_status st = upload_sites(ctx);
    if (st) return st;
    if (ctx->nslabs > 1 && (st = alloc_slab_rows(ctx, slab_capacity(ctx, thr)))) return st;
    if (ctx->p.gnUseOrientation) {
        CU(dzero(ctx, ctx->ka.d.rng_used, sizeof(int) * g.nranks));
        st = refill_rng(ctx, true);
    }
    return st;
}

mms_status mms_set_site_orientations(mms_ctx *ctx, int64_t n, const int32_t *gxyz, const double *rotmat9)
{
    if (!ctx || (n && (!gxyz || !rotmat9))) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    const Geo &g = ctx->ka.g, &G = ctx->gg;
    std::vector<std::pair<long long, int64_t>> kv;
    for (int64_t s = 0; s < n; s++) {
        long long x = gxyz[3 * s], y = gxyz[3 * s + 1], z = gxyz[3 * s + 2];
        if (x < 0 || y < 0 || z < 0 || x >= G.gx || y >= G.gy || z >= G.gz) return MMS_ERR_ARG;
        const long long zl = z - ctx->kz0;  // whole-domain z; another slab's cells are skipped
        if (zl < 0 || zl >= g.gz) continue;
        kv.push_back({cidx(g, x + 1, y + 1, zl + 1), s});
    }
    std::stable_sort(kv.begin(), kv.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
    ctx->inj_key.clear();
    ctx->inj_rot.clear();
    for (size_t i = 0; i < kv.size(); i++) {
        if (i > 0 && kv[i].first == kv[i - 1].first) continue;  // first listed wins
        ctx->inj_key.push_back(kv[i].first);
        for (int e = 0; e < 9; e++) ctx->inj_rot.push_back(rotmat9[9 * kv[i].second + e]);
    }
    DevPtrs &d = ctx->ka.d;
    drop_graph(ctx);
    dfree(ctx, d.inj_key);
    dfree(ctx, d.inj_rot);
    d.inj_key = nullptr;
    d.inj_rot = nullptr;
    size_t m = ctx->inj_key.size();
    mms_status st;
    if ((st = dalloc(ctx, &d.inj_key, m)) || (st = dalloc(ctx, &d.inj_rot, 9 * m))) return st;
    d.n_inj = (long long)m;
    if (m) {
        CU(h2d(ctx, d.inj_key, ctx->inj_key.data(), m * sizeof(long long)));
        CU(h2d(ctx, d.inj_rot, ctx->inj_rot.data(), 9 * m * sizeof(double)));
    }
    return MMS_OK;
}

// nsteps steps.  fold_fs: the last step runs the stencil that leaves
// per-tile fraction-solid sums, which are folded and copied to ctx->h_red
// before the closing control-block read, so one synchronisation covers
// both; *folded says whether that copy holds the fields as they stand (not
// after a stall, whose resumed steps come later).
static mms_status step_impl(mms_ctx *ctx, int nsteps, bool fold_fs, bool *folded)
{
    Range range("mms_step");
    *folded = false;
    if (!ctx || nsteps < 0) return MMS_ERR_ARG;
    if (ctx->nslabs > 1) {
        ctx->err = "a slab of a split domain steps with its group (mms_slab_group_step, mms_slab_launch)";
        return MMS_ERR_ARG;
    }
    cudaSetDevice(ctx->device);
    ctx->stepped = true;
    const int chunk = 256;
    int done = 0;
    mms_status st = MMS_OK;
    // the previous step call ended by reading the control block
    if (!ctx->ctl_known && (st = read_ctl(ctx))) return st;
    ctx->ctl_known = ctx->fs_part_valid = false;
    if (ctx->h_ctl->status) return (mms_status)ctx->h_ctl->status;
    unsigned long long ts0 = ctx->h_ctl->timestep;
    while (done < nsteps) {
        int n = std::min(chunk, nsteps - done);
        const long long nparts = stencil_parts(ctx->ka, ctx->tma);
        bool fold_now = fold_fs && done + n >= nsteps && nparts > 0;
        const int plain = n - (fold_now ? 1 : 0);  // steps without the sums
        if (ctx->use_graphs && !ctx->prof) {
            if ((st = ensure_graph(ctx))) return st;
            int s = 0;
            for (; s + GRAPH_STEPS <= plain; s += GRAPH_STEPS) {
                CU(cudaGraphLaunch(ctx->multi_graph, ctx->stream));
                ctx->launches += (uint64_t)ctx->step_graph_kernels * GRAPH_STEPS;
            }
            for (; s < plain; s++) {
                CU(cudaGraphLaunch(ctx->step_graph, ctx->stream));
                ctx->launches += ctx->step_graph_kernels;
            }
            if (fold_now) {
                CU(cudaGraphLaunch(ctx->sum_graph, ctx->stream));
                ctx->launches += ctx->step_graph_kernels;
            }
        } else {
            for (int s = 0; s < n; s++) ctx->launches += launch_one_step(ctx, 0, s >= plain);
        }
        if (fold_now && ctx->d_hctl) {
            // the fold kernel writes the sum and the control block to host
            // memory itself: the wait is the only thing left
            ctx->launches += launch_fold_fs_out(ctx->ka, nparts, ctx->stream, ctx->d_hred, ctx->d_hctl);
            CU(cudaGetLastError());
            Range wait("steps on the device");
            CU(cudaStreamSynchronize(ctx->stream));
            if (ctx->prof) ctx->prof->collect();
        } else {
            if (fold_now) ctx->launches += launch_fold_fs(ctx->ka, nparts, ctx->stream, ctx->h_red);
            CU(cudaGetLastError());
            Range wait("steps on the device");
            if ((st = read_ctl(ctx))) return st;
        }
        Ctl &c = *ctx->h_ctl;
        if (c.stall == STALL_ERROR) {
            ctx->err = mms_status_string((mms_status)c.status);
            return (mms_status)(c.status ? c.status : MMS_ERR_STATE);
        }
        if (c.stall == STALL_RNG) fold_now = false;
        *folded = fold_now;
        while (c.stall == STALL_RNG) {
            // a rank ran out of pre-drawn orientations at step stall_step:
            // refill, then resume that step at the activation stage
            Range stall("orientation refill and resume");
            if ((st = refill_rng(ctx, true))) return st;
            int zero = 0;
            CU(h2d(ctx, &ctx->ka.d.ctl->stall, &zero, sizeof(int)));
            ctx->launches += launch_one_step(ctx, 1);
            unsigned long long target = ts0 + done + n;
            if ((st = read_ctl(ctx))) return st;
            while (c.stall == 0 && c.timestep < target) {
                ctx->launches += launch_one_step(ctx, 0);
                if ((st = read_ctl(ctx))) return st;
            }
            if (c.stall == STALL_ERROR) return (mms_status)(c.status ? c.status : MMS_ERR_STATE);
        }
        done += n;
        if ((st = refill_rng(ctx, false))) return st;
    }
    ctx->ctl_known = true;
    ctx->fs_part_valid = *folded;
    return MMS_OK;
}

mms_status mms_step(mms_ctx *ctx, int nsteps)
{
    bool folded;
    return step_impl(ctx, nsteps, false, &folded);
}

// A sum of the fraction solid (each cell's fs capped at 1) or of ce over
// the domain, in the unit of `what` (computeFS, solid_volume,
// loop.c:173-183, growth.c:541-566).
static double reduce_scaled(const mms_ctx *ctx, mms_reduction what, double s)
{
    const mms_params &p = ctx->p;
    const Geo &g = ctx->ka.g;
    if (what == MMS_REDUCE_CE_SUM) return s;
    if (what == MMS_REDUCE_SOLID_VOLUME) return s * pow(p.cellSize, 3.0);
    return (s * pow(p.cellSize, 3.0)) / ((double)((long long)g.gx * g.gy * g.gz) * pow(p.cellSize, 3));
}

// The fs sum of the current fields: from the last step's per-tile sums when
// they are current, else a pass over the field.
static mms_status fs_sum(mms_ctx *ctx, double *s)
{
    const long long nparts = ctx->fs_part_valid ? stencil_parts(ctx->ka, ctx->tma) : 0;
    if (nparts > 0) {
        ctx->launches += launch_fold_fs(ctx->ka, nparts, ctx->stream, ctx->h_red);
        CU(cudaGetLastError());
        CU(cudaStreamSynchronize(ctx->stream));
        *s = *ctx->h_red;
        return MMS_OK;
    }
    ctx->launches += launch_reduce(ctx->ka, ctx->prec, 0, s, ctx->stream, ctx->h_red);
    CU(cudaGetLastError());
    return MMS_OK;
}

mms_status mms_step_reduce(mms_ctx *ctx, int nsteps, mms_reduction what, double *out)
{
    if (!ctx || !out) return MMS_ERR_ARG;
    const bool fs = what != MMS_REDUCE_CE_SUM;
    bool folded = false;
    mms_status st = step_impl(ctx, nsteps, fs, &folded);
    if (st) return st;
    if (folded) {
        *out = reduce_scaled(ctx, what, *ctx->h_red);
        return MMS_OK;
    }
    return mms_reduce(ctx, what, out);
}

mms_status mms_get_timestep(mms_ctx *ctx, uint64_t *timestep)
{
    if (!ctx || !timestep) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    mms_status st = read_ctl(ctx);
    if (st) return st;
    *timestep = ctx->h_ctl->timestep;
    return MMS_OK;
}

mms_status mms_get_num_grains(mms_ctx *ctx, int *num_grains)
{
    if (!ctx || !num_grains) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    mms_status st = read_ctl(ctx);
    if (st) return st;
    *num_grains = ctx->h_ctl->num_grains;
    return MMS_OK;
}

mms_status mms_download(mms_ctx *ctx, mms_field field, void *host)
{
    Range range("mms_download");
    if (!ctx || !host) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    const Geo &g = ctx->ka.g;
    const size_t N = (size_t)g.N;  // device layout
    mms_status st = read_ctl(ctx);
    if (st) return st;
    const int cur = (int)(ctx->h_ctl->timestep & 1ULL);
    DevPtrs &d = ctx->ka.d;
    switch (field) {
    case MMS_FIELD_CE:
    case MMS_FIELD_CL:
    case MMS_FIELD_FS: {
        if (ctx->prec == MMS_PREC_F64) {
            const void *src = field == MMS_FIELD_CE ? d.ce : (field == MMS_FIELD_CL ? d.cl[cur] : d.fs[cur]);
            CU(copy_out(ctx, host, src, sizeof(double)));
        } else {
            double *stg = (double *)stage_buffer(ctx, (size_t)g.rN * sizeof(double));
            if (!stg) return MMS_ERR_NOMEM;
            ctx->launches += launch_convert_ref(ctx->ka, ctx->prec, field, 0, stg, ctx->stream);
            CU(cudaMemcpyAsync(host, stg, (size_t)g.rN * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
            CU(cudaStreamSynchronize(ctx->stream));
        }
        return MMS_OK;
    }
    case MMS_FIELD_GR:
        CU(copy_out(ctx, host, d.gr, sizeof(int)));
        return MMS_OK;
    case MMS_FIELD_OGR: {
        int *tmp;
        if ((st = dalloc(ctx, &tmp, N))) return st;
        CU(cudaMemcpyAsync(tmp, d.gr, N * sizeof(int), cudaMemcpyDeviceToDevice, ctx->stream));
        ctx->launches += launch_mask_captured(ctx->ka, tmp, 0, ctx->stream);
        CU(copy_out(ctx, host, tmp, sizeof(int)));
        dfree(ctx, tmp);
        return MMS_OK;
    }
    case MMS_FIELD_DC:
        CU(copy_out(ctx, host, d.dc, sizeof(Dc3)));
        return MMS_OK;
    case MMS_FIELD_CURV:
        if (!d.curv) {
            std::memset(host, 0, (size_t)g.rN * sizeof(double));
            return MMS_OK;
        }
        CU(copy_out(ctx, host, d.curv, sizeof(double)));
        return MMS_OK;
    case MMS_FIELD_D:
    case MMS_FIELD_TEMPERATURE: {
        double *tmp;
        if ((st = dalloc(ctx, &tmp, N))) return st;
        if (field == MMS_FIELD_D) {
            ctx->launches += launch_compute_d(ctx->ka, ctx->prec, tmp, ctx->stream);
            ctx->launches += launch_mask_captured(ctx->ka, tmp, 1, ctx->stream);
        } else {
            ctx->launches += launch_fill_temperature(ctx->ka, tmp, ctx->stream);
            // FP32 AM form: the halo columns, which no kernel of a step reads,
            // from the tables of the current step
            if (ctx->ka.p.temp_mode == 2 && ctx->prec == MMS_PREC_F32)
                ctx->launches += launch_am_halo_fill(ctx->ka, am_params(ctx->p), tmp, ctx->stream);
        }
        CU(copy_out(ctx, host, tmp, sizeof(double)));
        dfree(ctx, tmp);
        return MMS_OK;
    }
    case MMS_FIELD_NUC_THRESHOLD: {
        float *t = (float *)host;
        for (long long c = 0; c < g.rN; c++) t[c] = INFINITY;
        for (size_t s = 0; s < ctx->site_cell.size(); s++) t[dev_to_ref(g, ctx->site_cell[s])] = ctx->site_thr[s];
        return MMS_OK;
    }
    case MMS_FIELD_MOLD: {
        std::vector<signed char> m = make_mold(g);
        std::memcpy(host, m.data(), m.size());
        return MMS_OK;
    }
    }
    return MMS_ERR_ARG;
}

mms_status mms_upload(mms_ctx *ctx, mms_field field, const void *host)
{
    Range range("mms_upload");
    if (!ctx || !host) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    ctx->fs_part_valid = false;
    const Geo &g = ctx->ka.g;
    const size_t N = (size_t)g.N;
    mms_status st;
    DevPtrs &d = ctx->ka.d;
    switch (field) {
    case MMS_FIELD_CE:
    case MMS_FIELD_CL:
    case MMS_FIELD_FS: {
        // cl and fs are written to both step buffers (the stencil writes
        // only interior cells of its output buffer)
        if ((st = read_ctl(ctx))) return st;
        const int cur = (int)(ctx->h_ctl->timestep & 1ULL);
        if (ctx->prec == MMS_PREC_F64) {
            void *dst = field == MMS_FIELD_CE ? d.ce : (field == MMS_FIELD_CL ? d.cl[cur] : d.fs[cur]);
            CU(copy_in(ctx, dst, host, sizeof(double)));
            if (field != MMS_FIELD_CE) {
                void *other = field == MMS_FIELD_CL ? d.cl[cur ^ 1] : d.fs[cur ^ 1];
                CU(cudaMemcpyAsync(other, dst, N * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
                CU(cudaStreamSynchronize(ctx->stream));
            }
            return MMS_OK;
        }
        // FP32 form: the doubles land in the staging buffer and are
        // converted from the reference layout on the device
        double *stg = (double *)stage_buffer(ctx, (size_t)g.rN * sizeof(double));
        if (!stg) return MMS_ERR_NOMEM;
        CU(cudaMemcpyAsync(stg, host, (size_t)g.rN * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        ctx->launches += launch_convert_ref(ctx->ka, ctx->prec, field, 1, stg, ctx->stream);
        CU(cudaStreamSynchronize(ctx->stream));
        return MMS_OK;
    }
    case MMS_FIELD_GR:
        CU(copy_in(ctx, d.gr, host, sizeof(int)));
        return MMS_OK;
    case MMS_FIELD_DC:
        CU(copy_in(ctx, d.dc, host, sizeof(Dc3)));
        return MMS_OK;
    case MMS_FIELD_NUC_THRESHOLD: {
        std::vector<float> thr((const float *)host, (const float *)host + g.rN);
        extract_sites(ctx, thr);
        return upload_sites(ctx);
    }
    default:
        return MMS_ERR_ARG;
    }
}

mms_status mms_reduce(mms_ctx *ctx, mms_reduction what, double *out)
{
    Range range("mms_reduce");
    if (!ctx || !out) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    double s = 0;
    if (what == MMS_REDUCE_CE_SUM) {
        ctx->launches += launch_reduce(ctx->ka, ctx->prec, MMS_REDUCE_CE_SUM, &s, ctx->stream, ctx->h_red);
        CU(cudaGetLastError());
    } else {
        mms_status st = fs_sum(ctx, &s);
        if (st) return st;
    }
    *out = reduce_scaled(ctx, what, s);
    return MMS_OK;
}

mms_status mms_get_grains(mms_ctx *ctx, int first, int count, mms_grain *out)
{
    if (!ctx || !out || first < 0 || count < 0) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    mms_status st = sync_grains(ctx);
    if (st) return st;
    for (int i = 0; i < count; i++) {
        int gi = first + i;
        if (gi < (int)ctx->grains.size()) out[i] = ctx->grains[gi];
        else std::memset(&out[i], 0, sizeof(mms_grain));
    }
    return MMS_OK;
}

// output_grains (grain.c:751-833)
mms_status mms_output_grains(mms_ctx *ctx, const char *path, mms_grain_summary *out)
{
    if (!ctx) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    mms_status st = sync_grains(ctx);
    if (st) return st;
    const Geo &g = ctx->ka.g;
    const mms_params &p = ctx->p;
    int ng = ctx->h_ctl->num_grains;
    std::vector<int> gr((size_t)g.rN);
    CU(copy_out(ctx, gr.data(), ctx->ka.d.gr, sizeof(int)));
    std::vector<size_t> sizes((size_t)ng + 1, 0);
    for (long long k = 1; k <= g.gz; k++)
        for (long long j = 1; j <= g.gy; j++)
            for (long long i = 1; i <= g.gx; i++) {
                int v = gr[rcidx(g, i, j, k)];
                if (v > 0 && v <= ng) sizes[v]++;
            }
    size_t minSize = sizes[1], maxSize = sizes[1], avgSize = 0, zeroCount = 0;
    double cellVolume = pow(p.cellSize * 1000, 3.0);
    FILE *fp = nullptr;
    if (path) {
        fp = std::fopen(path, "w");
        if (!fp) {
            ctx->err = std::string("Unable to open grain file ") + path;
            return MMS_ERR_IO;
        }
        std::fprintf(fp, "Number,Nuc Timestep,Nuc Time,Nuc Threshold,X,Y,Z,CellX,CellY,CellZ,Rot1,Rot2,Rot3,"
                         "Rotation Matrix,Size mm^3\n");
    }
    for (int i = 1; i < ng; i++) {
        const mms_grain &gg = ctx->grains[i];
        if (fp) {
            size_t cx, cy, cz;
            real2cell(p, gg.nuc_x, gg.nuc_y, gg.nuc_z, &cx, &cy, &cz);
            std::fprintf(fp,
                         "%d,%lu,%lg,%lg,%lg,%lg,%lg,%lu,%lu,%lu,%lg,%lg,%lg,[[%lg %lg %lg][%lg %lg %lg][%lg %lg %lg]],%lg\n",
                         i, (unsigned long)gg.nuc_timestep, gg.nuc_timestep * p.ts_delt, gg.nuc_threshold, gg.nuc_x,
                         gg.nuc_y, gg.nuc_z, cx, cy, cz, gg.rotang[0], gg.rotang[1], gg.rotang[2], gg.rotmat[0][0],
                         gg.rotmat[0][1], gg.rotmat[0][2], gg.rotmat[1][0], gg.rotmat[1][1], gg.rotmat[1][2],
                         gg.rotmat[2][0], gg.rotmat[2][1], gg.rotmat[2][2], sizes[i] * cellVolume);
        }
        if (sizes[i] < minSize) minSize = sizes[i];
        if (sizes[i] > maxSize) maxSize = sizes[i];
        avgSize += sizes[i];
        if (sizes[i] == 0) zeroCount++;
    }
    if (fp) std::fclose(fp);
    if (out) {
        out->num_grains = ng - 1;
        out->min_mm3 = minSize * cellVolume;
        out->max_mm3 = maxSize * cellVolume;
        out->avg_mm3 = ((double)avgSize / ((double)((ng - 1) - zeroCount)) * cellVolume);
    }
    return MMS_OK;
}

// loop (loop.c:185-271): screen lines every ScreenPFreq, termination by
// FinishTime or FsFinish, grain summary at the end.  verbose: 0 quiet,
// 1 screen output, 2 screen output in interactive mode (-i).
mms_status mms_run(mms_ctx *ctx, int verbose)
{
    Range range("mms_run");
    if (!ctx) return MMS_ERR_ARG;
    const mms_params &p = ctx->p;
    const char *leader = (verbose == 2) ? "        \r" : "";
    const char *tailer = (verbose == 2) ? "" : "\n";
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    double t0 = tv.tv_sec + ((double)tv.tv_usec * 1.0e-6);
    auto screen = [&](double fs) {
        gettimeofday(&tv, nullptr);
        double t = tv.tv_sec + ((double)tv.tv_usec * 1.0e-6);
        int ng = 0;
        mms_get_num_grains(ctx, &ng);
        uint64_t ts = 0;
        mms_get_timestep(ctx, &ts);
        std::printf("%s%10g  %10g  %8.4lf%% %8d  %s \n", leader, t - t0, ts * p.ts_delt, 100.0 * fs, ng - 1, tailer);
        std::fflush(stdout);
    };
    if (verbose && p.screenpfreq > 0) {
        std::printf("\n%10s  %10s   %8s  %8s\n", "Wall Time", "Sim Time", "Fraction", "Grain NO");
        std::printf("%10s  %10s   %8s\n", "(sec)  ", "(sec)  ", "Solid");
        screen(0.0);
    }
    double fs = 0.0;
    mms_status st;
    uint64_t ts = 0;
    if ((st = mms_get_timestep(ctx, &ts))) return st;
    // data files as writeData (loop.c:116-128): VTK or XDMF, at the start,
    // every DataWriteFreq steps from DataWriteStart, and at the end
    const bool data = p.data_write_freq > 0 && (p.vis_format == 1 || p.vis_format == 2);
    auto write_data = [&]() -> mms_status {
        return p.vis_format == 1 ? mms_write_vtk(ctx, nullptr) : mms_write_xdmf(ctx, nullptr);
    };
    if (data && ts == 0 && (st = write_data())) return st;
    for (;;) {
        // run to the next screen step, or to FinishTime if that comes first
        uint64_t n = (p.screenpfreq > 0) ? (uint64_t)p.screenpfreq - (ts % (uint64_t)p.screenpfreq) : (1ULL << 30);
        if (data) n = std::min<uint64_t>(n, (uint64_t)p.data_write_freq - (ts % (uint64_t)p.data_write_freq));
        if (p.checkpoint_freq > 0)
            n = std::min<uint64_t>(n, (uint64_t)p.checkpoint_freq - (ts % (uint64_t)p.checkpoint_freq));
        if (p.finish_time) {
            // first t with t*ts_delt >= finish_time (checkDone, loop.c:155-156)
            uint64_t t = (uint64_t)std::floor(p.finish_time / p.ts_delt);
            while (t > 0 && ((t - 1) * p.ts_delt) >= p.finish_time) t--;
            while ((t * p.ts_delt) < p.finish_time) t++;
            if (t <= ts) t = ts + 1;
            n = std::min<uint64_t>(n, t - ts);
        }
        if (n > (1ULL << 30)) n = 1ULL << 30;
        // a chunk that ends on a screen step also sums the fraction solid
        const bool screen_step = p.screenpfreq > 0 && (ts + n) % (uint64_t)p.screenpfreq == 0;
        double fs_now = fs;
        if (screen_step) st = mms_step_reduce(ctx, (int)n, MMS_REDUCE_FS_FRACTION, &fs_now);
        else st = mms_step(ctx, (int)n);
        if (st) return st;
        ts += n;
        if (data && ts >= (uint64_t)p.data_write_start && ts % (uint64_t)p.data_write_freq == 0 &&
            (st = write_data()))
            return st;
        if (screen_step) {
            fs = fs_now;
            if (verbose) screen(fs);
        }
        // writeCheckpoint (loop.c:244-247), in this library's raw format
        if (p.checkpoint_freq > 0 && ts % (uint64_t)p.checkpoint_freq == 0 &&
            (st = mms_checkpoint_save(ctx, MMS_CHECKPOINT_FILE)))
            return st;
        bool done = false;
        if (p.finish_time && ((ts * p.ts_delt) >= p.finish_time)) {
            done = true;
            if (verbose) std::printf("\nAuto-Finish time met.\n");
        }
        if (fs >= p.fs_finish) {
            if (verbose) std::printf("\nSolid Fraction termination condition met.\n");
            done = true;
        }
        if (done) break;
    }
    if (data && ts % (uint64_t)p.data_write_freq != 0 && (st = write_data())) return st;
    mms_grain_summary s;
    char path[512];
    std::snprintf(path, sizeof path, "%s_grains.csv", p.basefilename);
    if ((st = mms_output_grains(ctx, verbose ? path : nullptr, &s))) return st;
    if (verbose) {
        std::printf("%d grains.  Min: %lg mm^3   Max: %lg mm^3   Average:  %lg mm^3\n", s.num_grains, s.min_mm3,
                    s.max_mm3, s.avg_mm3);
        std::printf("\nSimulation complete.  Shutting down.\n");
        std::fflush(stdout);
    }
    return MMS_OK;
}

}  // extern "C"

// ============================================================ adjoint (host)
namespace {

size_t elem_size(const mms_ctx *ctx) { return ctx->prec == MMS_PREC_F32 ? sizeof(float) : sizeof(double); }

void adj_stop_recording(mms_ctx *ctx)
{
    DevPtrs &d = ctx->ka.d;
    if (d.rec_flags) {
        d.rec_flags = nullptr;
        d.rec_curv = nullptr;
        d.rec_cap = 0;
        drop_graph(ctx);
    }
}

void adj_free(mms_ctx *ctx)
{
    adj_stop_recording(ctx);
    dfree(ctx, ctx->adj.flags);
    dfree(ctx, ctx->adj.curv);
    dfree(ctx, ctx->adj.ckpt);
    ctx->adj = mms_ctx::AdjRec{};
}

// state slot s of a buffer of 3 x N x es per slot
char *state_slot(char *base, long long s, int f, size_t N, size_t es) { return base + ((size_t)s * 3 + f) * N * es; }

mms_status adj_save_ckpt(mms_ctx *ctx, long long idx, unsigned long long ts)
{
    const size_t N = (size_t)ctx->ka.g.N, es = elem_size(ctx);
    const int b = (int)(ts & 1ULL);
    const void *src[3] = {ctx->ka.d.ce, ctx->ka.d.cl[b], ctx->ka.d.fs[b]};
    for (int f = 0; f < 3; f++)
        CU(cudaMemcpyAsync(state_slot(ctx->adj.ckpt, idx, f, N, es), src[f], N * es, cudaMemcpyDeviceToDevice,
                           ctx->stream));
    return MMS_OK;
}

// Phys with Dliq, part_coef and the Gibbs-Thomson coefficient scaled, each
// derived constant computed as mms_create computes it.
Phys scaled_phys(const mms_ctx *ctx, const double scale[3])
{
    const mms_params &p = ctx->p;
    Phys ph = ctx->ka.p;
    const double dtx = p.ts_delt / (p.cellSize * p.cellSize);
    const double Dliq = p.Dliq * scale[0], k = p.part_coef * scale[1];
    ph.rl = Dliq * dtx;
    ph.D_xt = (Dliq / p.cellSize / p.cellSize) * p.ts_delt;
    ph.k_inv = 1.0 / k;
    ph.km = 1.0 - k;
    ph.km_inv = 1.0 / ph.km;
    ph.gibbs = p.gibbs_coef * scale[2];
    return ph;
}

}  // namespace

extern "C" {

mms_status mms_adjoint_release(mms_ctx *ctx)
{
    if (!ctx) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    adj_free(ctx);
    return MMS_OK;
}

mms_status mms_adjoint_record(mms_ctx *ctx, int nsteps, int checkpoint_every)
{
    Range range("mms_adjoint_record");
    if (ctx) ctx->ctl_known = ctx->fs_part_valid = false;
    if (!ctx || nsteps < 1 || checkpoint_every < 1 || ctx->nslabs > 1) return MMS_ERR_ARG;
    if (ctx->ka.p.temp_mode == 2) {
        ctx->err = "the adjoint supports the analytic temperature models only";
        return MMS_ERR_ARG;
    }
    cudaSetDevice(ctx->device);
    mms_status st = read_ctl(ctx);
    if (st) return st;
    if (ctx->h_ctl->status) return (mms_status)ctx->h_ctl->status;
    adj_free(ctx);
    const size_t N = (size_t)ctx->ka.g.N, es = elem_size(ctx);
    mms_ctx::AdjRec &r = ctx->adj;
    r.t0 = ctx->h_ctl->timestep;
    r.nrec = nsteps;
    r.every = checkpoint_every;
    r.nckpt = (nsteps + checkpoint_every - 1) / checkpoint_every;
    if ((st = dalloc(ctx, &r.flags, (size_t)nsteps * N)) ||
        (ctx->p.tip_curv && (st = dalloc(ctx, &r.curv, (size_t)nsteps * N))) ||
        (st = dalloc(ctx, &r.ckpt, (size_t)r.nckpt * 3 * N * es))) {
        adj_free(ctx);
        return st;
    }
    if ((st = adj_save_ckpt(ctx, 0, r.t0))) return st;
    DevPtrs &d = ctx->ka.d;
    d.rec_flags = r.flags;
    d.rec_curv = r.curv;
    d.rec_t0 = r.t0;
    d.rec_cap = nsteps;
    drop_graph(ctx);
    long long done = 0;
    while (done < nsteps) {
        int n = (int)std::min<long long>(checkpoint_every, nsteps - done);
        if ((st = mms_step(ctx, n))) {
            adj_free(ctx);
            return st;
        }
        done += n;
        if (done < nsteps && (st = adj_save_ckpt(ctx, done / checkpoint_every, r.t0 + done))) return st;
    }
    adj_stop_recording(ctx);
    CU(cudaStreamSynchronize(ctx->stream));
    return MMS_OK;
}

mms_status mms_adjoint_replay_loss(mms_ctx *ctx, const double *target_ce, const double scale[3], double *loss)
{
    if (!ctx || !target_ce || !scale || !loss) return MMS_ERR_ARG;
    if (!ctx->adj.nrec) return MMS_ERR_STATE;
    cudaSetDevice(ctx->device);
    ctx->fs_part_valid = false;
    const Geo &g = ctx->ka.g;
    const size_t N = (size_t)g.N, es = elem_size(ctx);
    const mms_ctx::AdjRec &r = ctx->adj;
    const Phys ph = scaled_phys(ctx, scale);
    char *buf = nullptr;
    double *tgt = nullptr, *partial = nullptr, *dl = nullptr;
    mms_status st;
    auto cleanup = [&]() {
        cudaStreamSynchronize(ctx->stream);
        dfree(ctx, buf);
        dfree(ctx, tgt);
        dfree(ctx, partial);
        dfree(ctx, dl);
    };
    if ((st = dalloc(ctx, &buf, 2 * 3 * N * es)) || (st = dalloc(ctx, &tgt, N)) ||
        (st = dalloc(ctx, &partial, (size_t)adj_nblocks(g))) || (st = dalloc(ctx, &dl, 1))) {
        cleanup();
        return st;
    }
    cudaError_t e = copy_in(ctx, tgt, target_ce, sizeof(double));
    for (int b = 0; b < 2 && e == cudaSuccess; b++)
        for (int f = 0; f < 3 && e == cudaSuccess; f++)
            e = cudaMemcpyAsync(state_slot(buf, b, f, N, es), state_slot(r.ckpt, 0, f, N, es), N * es,
                                cudaMemcpyDeviceToDevice, ctx->stream);
    int cur = 0;
    for (long long s = 0; s < r.nrec && e == cudaSuccess; s++) {
        const void *x0[3] = {state_slot(buf, cur, 0, N, es), state_slot(buf, cur, 1, N, es),
                             state_slot(buf, cur, 2, N, es)};
        void *x1[3] = {state_slot(buf, 1 - cur, 0, N, es), state_slot(buf, 1 - cur, 1, N, es),
                       state_slot(buf, 1 - cur, 2, N, es)};
        launch_replay(g, ph, ctx->prec, x0, x1, r.flags + (size_t)s * N, r.curv ? r.curv + (size_t)s * N : nullptr,
                      r.t0 + s + 1, ctx->stream);
        cur = 1 - cur;
    }
    const double off = ctx->prec == MMS_PREC_F32 ? ctx->p.Cinit : 0.0;
    if (e == cudaSuccess) {
        launch_adj_terminal(g, ctx->prec, off, state_slot(buf, cur, 0, N, es), tgt, nullptr, nullptr, nullptr,
                            partial, dl, ctx->stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(loss, dl, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cleanup();
    if (e != cudaSuccess) {
        ctx->err = std::string("adjoint replay: ") + cudaGetErrorString(e);
        return MMS_ERR_CUDA;
    }
    return MMS_OK;
}

mms_status mms_adjoint_gradient(mms_ctx *ctx, const double *target_ce, mms_adjoint_result *out)
{
    Range range("mms_adjoint_gradient");
    if (!ctx || !target_ce || !out) return MMS_ERR_ARG;
    if (!ctx->adj.nrec) return MMS_ERR_STATE;
    cudaSetDevice(ctx->device);
    ctx->fs_part_valid = false;
    const Geo &g = ctx->ka.g;
    const size_t N = (size_t)g.N, es = elem_size(ctx);
    const mms_ctx::AdjRec &r = ctx->adj;
    const Phys &ph = ctx->ka.p;
    const int nb = adj_nblocks(g);
    char *seg = nullptr, *lam = nullptr;
    double *tgt = nullptr, *partial = nullptr, *acc = nullptr;
    mms_status st;
    auto cleanup = [&]() {
        cudaStreamSynchronize(ctx->stream);
        dfree(ctx, seg);
        dfree(ctx, lam);
        dfree(ctx, tgt);
        dfree(ctx, partial);
        dfree(ctx, acc);
    };
    // acc: ADJ_SLOTS gradient sums, then the loss
    if ((st = dalloc(ctx, &seg, (size_t)(r.every + 1) * 3 * N * es)) || (st = dalloc(ctx, &lam, 6 * N * es)) ||
        (st = dalloc(ctx, &tgt, N)) || (st = dalloc(ctx, &partial, (size_t)nb * ADJ_SLOTS)) ||
        (st = dalloc(ctx, &acc, ADJ_SLOTS + 1))) {
        cleanup();
        return st;
    }
    // adjoint buffers: lce, lcl[2], lfs[2], nu
    char *lce = lam, *lcl[2] = {lam + N * es, lam + 2 * N * es}, *lfs[2] = {lam + 3 * N * es, lam + 4 * N * es},
         *nu = lam + 5 * N * es;
    cudaError_t e = copy_in(ctx, tgt, target_ce, sizeof(double));
    const double off = ctx->prec == MMS_PREC_F32 ? ctx->p.Cinit : 0.0;
    int lc = 0;
    for (long long sg = r.nckpt - 1; sg >= 0 && e == cudaSuccess; sg--) {
        const long long s0 = sg * r.every, s1 = std::min<long long>(s0 + r.every, r.nrec), L = s1 - s0;
        // every slot starts as the checkpoint (halo cells never change)
        for (long long l = 0; l <= L && e == cudaSuccess; l++)
            for (int f = 0; f < 3 && e == cudaSuccess; f++)
                e = cudaMemcpyAsync(state_slot(seg, l, f, N, es), state_slot(r.ckpt, sg, f, N, es), N * es,
                                    cudaMemcpyDeviceToDevice, ctx->stream);
        for (long long l = 0; l < L; l++) {
            const void *x0[3] = {state_slot(seg, l, 0, N, es), state_slot(seg, l, 1, N, es),
                                 state_slot(seg, l, 2, N, es)};
            void *x1[3] = {state_slot(seg, l + 1, 0, N, es), state_slot(seg, l + 1, 1, N, es),
                           state_slot(seg, l + 1, 2, N, es)};
            const size_t s = (size_t)(s0 + l);
            launch_replay(g, ph, ctx->prec, x0, x1, r.flags + s * N, r.curv ? r.curv + s * N : nullptr,
                          r.t0 + s + 1, ctx->stream);
        }
        if (sg == r.nckpt - 1)
            launch_adj_terminal(g, ctx->prec, off, state_slot(seg, L, 0, N, es), tgt, lce, lcl[lc], lfs[lc],
                                partial, acc + ADJ_SLOTS, ctx->stream);
        for (long long l = L - 1; l >= 0; l--) {
            const void *x0[3] = {state_slot(seg, l, 0, N, es), state_slot(seg, l, 1, N, es),
                                 state_slot(seg, l, 2, N, es)};
            const size_t s = (size_t)(s0 + l);
            launch_adj_step(g, ph, ctx->prec, x0, state_slot(seg, l + 1, 0, N, es), r.flags + s * N,
                            r.curv ? r.curv + s * N : nullptr, lce, lcl[lc], lfs[lc], lcl[1 - lc], lfs[1 - lc], nu,
                            partial, acc, r.t0 + s + 1, ctx->stream);
            lc = 1 - lc;
        }
        if (e == cudaSuccess) e = cudaGetLastError();
    }
    double h[ADJ_SLOTS + 1] = {};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, acc, sizeof h, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cleanup();
    if (e != cudaSuccess) {
        ctx->err = std::string("adjoint: ") + cudaGetErrorString(e);
        return MMS_ERR_CUDA;
    }
    // chain rule to the deck parameters: rl = Dliq dt/dx^2, D_xt = Dliq/dx/dx dt,
    // km = 1 - k, km_inv = 1/(1 - k), k_inv = 1/k
    const mms_params &p = ctx->p;
    const double dtx = p.ts_delt / (p.cellSize * p.cellSize);
    const double k = p.part_coef, km = 1.0 - k;
    out->loss = h[ADJ_SLOTS];
    out->dL_dDliq = (h[0] + h[1]) * dtx;
    out->dL_dpart_coef = -h[2] + h[3] / (km * km) - h[4] / (k * k);
    out->dL_dgibbs = h[5];
    out->steps = r.nrec;
    return MMS_OK;
}

}  // extern "C"

// ============================================================ batched domains
// Many independent domains stepped together: one CUDA graph per step holds
// every domain's nucleation and activation (parallel branches), ONE
// persistent stencil launch over the tiles of all domains, and every
// domain's list and capture (parallel branches).
struct mms_batch {
    std::vector<mms_ctx *> doms;
    int prec = MMS_PREC_F64;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> ev_fork, ev_join;
    void *items = nullptr;  // device array of batch items
    long long total_tiles = 0;
    // prefix sums of the small kernels' blocks per domain (nucleation,
    // activation, list, capture), n + 1 each, on the device
    int *begin = nullptr;
    int totals[4] = {0, 0, 0, 0};
    int graph_totals[4] = {-1, -1, -1, -1};
    int cpt = 1, zc = 0, grid = 0;
    cudaGraphExec_t graph = nullptr;
    int graph_kernels = 0;
    uint64_t launches = 0;
    std::string err;
};

namespace {

void batch_drop_graph(mms_batch *b)
{
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
}

// Kernel arguments of every domain (sites and tables can be replaced
// between calls) and the small kernels' block prefixes; the step graph is
// dropped when a launch's block total changed.
mms_status batch_refresh(mms_batch *b)
{
    const size_t nd = b->doms.size(), ib = batch_item_bytes();
    if (!b->items) return MMS_OK;
    std::vector<unsigned char> host(ib * nd);
    std::vector<int> begin(4 * (nd + 1), 0);
    long long tiles = 0;
    for (size_t i = 0; i < nd; i++) {
        mms_ctx *ctx = b->doms[i];
        tiles += fill_batch_item(host.data() + ib * i, ctx->ka, ctx->tma, tiles);
        for (int w = 0; w < 4; w++) begin[w * (nd + 1) + i + 1] = begin[w * (nd + 1) + i] + batch_blocks(ctx->ka, w);
    }
    if (!b->begin && cudaMalloc(&b->begin, sizeof(int) * begin.size()) != cudaSuccess) {
        b->err = "cudaMalloc of the batch prefixes failed";
        return MMS_ERR_NOMEM;
    }
    if (cudaMemcpyAsync(b->items, host.data(), host.size(), cudaMemcpyHostToDevice, b->stream) != cudaSuccess ||
        cudaMemcpyAsync(b->begin, begin.data(), sizeof(int) * begin.size(), cudaMemcpyHostToDevice, b->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess)
        return MMS_ERR_CUDA;
    for (int w = 0; w < 4; w++) {
        b->totals[w] = begin[w * (nd + 1) + nd];
        if (b->totals[w] != b->graph_totals[w]) batch_drop_graph(b);
    }
    return MMS_OK;
}

mms_status batch_build_items(mms_batch *b)
{
    const size_t ib = batch_item_bytes();
    std::vector<unsigned char> host(ib * b->doms.size());
    long long tiles = 0;
    for (size_t i = 0; i < b->doms.size(); i++) {
        mms_ctx *ctx = b->doms[i];
        ctx->tma.cpt = b->cpt;
        ctx->tma.zc = b->zc;
        if (!make_tma(ctx->ka, ctx->prec, ctx->tma)) {
            b->err = "TMA descriptors could not be encoded for a batched domain";
            return MMS_ERR_CUDA;
        }
        drop_graph(ctx);
        tiles += fill_batch_item(host.data() + ib * i, ctx->ka, ctx->tma, tiles);
    }
    if (b->items) cudaFree(b->items);
    b->items = nullptr;
    if (cudaMalloc(&b->items, host.size()) != cudaSuccess) {
        b->err = "cudaMalloc of the batch items failed";
        return MMS_ERR_NOMEM;
    }
    if (cudaMemcpyAsync(b->items, host.data(), host.size(), cudaMemcpyHostToDevice, b->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess)
        return MMS_ERR_CUDA;
    b->total_tiles = tiles;
    b->grid = batch_grid(b->prec, b->cpt);
    batch_drop_graph(b);
    return batch_refresh(b);
}

// One step of every domain, on b->stream (captured into the step graph):
// AM temperatures as parallel branches, then one launch each of nucleation
// and activation over all domains, curvature branches (TipCurvature decks),
// the persistent stencil, and one launch each of list and capture.
int batch_launch_step(mms_batch *b)
{
    int n = 0;
    const int nd = (int)b->doms.size();
    auto branches = [&](auto &&fn) {
        bool any = false;
        for (int i = 0; i < nd; i++) {
            mms_ctx *ctx = b->doms[i];
            if (!fn(ctx, nullptr)) continue;
            if (!any) cudaEventRecord(b->ev_fork[0], b->stream);
            any = true;
            cudaStreamWaitEvent(b->side[i], b->ev_fork[0], 0);
            n += fn(ctx, b->side[i]);
            cudaEventRecord(b->ev_join[i], b->side[i]);
            cudaStreamWaitEvent(b->stream, b->ev_join[i], 0);
        }
    };
    // fn(ctx, nullptr) asks whether the domain has such work
    branches([&](mms_ctx *ctx, cudaStream_t s) -> int {
        if (!ctx->p.am) return 0;
        return s ? launch_temp_am(ctx->ka, am_params(ctx->p), ctx->prec, s, nullptr, ctx->am_rows) : 1;
    });
    const int *bg = b->begin;
    n += launch_small_batch(0, b->items, bg, nd, b->totals[0], b->prec, b->stream);
    n += launch_small_batch(1, b->items, bg + (nd + 1), nd, b->totals[1], b->prec, b->stream);
    branches([&](mms_ctx *ctx, cudaStream_t s) -> int {
        if (!ctx->p.tip_curv) return 0;
        return s ? launch_curv(ctx->ka, ctx->prec, s) : 1;
    });
    n += launch_stencil_batch(b->items, nd, b->total_tiles, b->prec, b->cpt, b->grid, b->stream);
    n += launch_small_batch(2, b->items, bg + 2 * (nd + 1), nd, b->totals[2], b->prec, b->stream);
    n += launch_small_batch(3, b->items, bg + 3 * (nd + 1), nd, b->totals[3], b->prec, b->stream);
    return n;
}

mms_status batch_ensure_graph(mms_batch *b)
{
    if (b->graph) return MMS_OK;
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return MMS_ERR_CUDA;
    int n = batch_launch_step(b);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        b->graph = nullptr;
        b->err = std::string("batch graph: ") + cudaGetErrorString(e);
        return MMS_ERR_CUDA;
    }
    b->graph_kernels = n;
    for (int w = 0; w < 4; w++) b->graph_totals[w] = b->totals[w];
    return MMS_OK;
}

// Brings a domain whose step stalled on orientation draws up to `target`.
mms_status batch_resume(mms_ctx *ctx, unsigned long long target)
{
    mms_status st;
    Ctl &c = *ctx->h_ctl;
    while (c.stall == STALL_RNG) {
        if ((st = refill_rng(ctx, true))) return st;
        int zero = 0;
        CU(h2d(ctx, &ctx->ka.d.ctl->stall, &zero, sizeof(int)));
        ctx->launches += launch_one_step(ctx, 1);
        if ((st = read_ctl(ctx))) return st;
        while (c.stall == 0 && c.timestep < target) {
            ctx->launches += launch_one_step(ctx, 0);
            if ((st = read_ctl(ctx))) return st;
        }
    }
    if (c.stall == STALL_ERROR) {
        ctx->err = mms_status_string((mms_status)c.status);
        return (mms_status)(c.status ? c.status : MMS_ERR_STATE);
    }
    return MMS_OK;
}

}  // namespace

extern "C" {

mms_status mms_batch_destroy(mms_batch *b)
{
    if (!b) return MMS_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_drop_graph(b);
    for (mms_ctx *ctx : b->doms) mms_destroy(ctx);
    if (b->items) cudaFree(b->items);
    if (b->begin) cudaFree(b->begin);
    for (cudaStream_t s : b->side) cudaStreamDestroy(s);
    for (cudaEvent_t e : b->ev_fork) cudaEventDestroy(e);
    for (cudaEvent_t e : b->ev_join) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return MMS_OK;
}

mms_status mms_batch_create(int n, const mms_params *params, mms_batch **out)
{
    if (!out || n < 1 || !params) return MMS_ERR_ARG;
    *out = nullptr;
    for (int i = 1; i < n; i++)
        if (params[i].precision != params[0].precision || params[i].device != params[0].device) return MMS_ERR_ARG;
    mms_batch *b = new mms_batch();
    b->prec = params[0].precision == MMS_PREC_F32 ? MMS_PREC_F32 : MMS_PREC_F64;
    b->device = params[0].device;
    for (int i = 0; i < n; i++) {
        mms_ctx *ctx = nullptr;
        mms_status st = mms_create(&params[i], &ctx);
        if (st) {
            mms_batch_destroy(b);
            return st;
        }
        b->doms.push_back(ctx);
    }
    cudaSetDevice(b->device);
    cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    b->side.resize(n);
    b->ev_join.resize(n);
    b->ev_fork.resize(2);
    for (int i = 0; i < n; i++) {
        cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking);
        cudaEventCreateWithFlags(&b->ev_join[i], cudaEventDisableTiming);
    }
    for (auto &e : b->ev_fork) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    for (mms_ctx *ctx : b->doms) mms_set_stream(ctx, b->stream);
    mms_status st = batch_build_items(b);
    if (st) {
        mms_batch_destroy(b);
        return st;
    }
    *out = b;
    return MMS_OK;
}

int mms_batch_size(const mms_batch *b) { return b ? (int)b->doms.size() : 0; }

mms_ctx *mms_batch_domain(mms_batch *b, int i)
{
    if (!b || i < 0 || i >= (int)b->doms.size()) return nullptr;
    return b->doms[i];
}

mms_status mms_batch_step(mms_batch *b, int nsteps)
{
    Range range("mms_batch_step");
    if (!b || nsteps < 0) return MMS_ERR_ARG;
    cudaSetDevice(b->device);
    mms_status st;
    const size_t nd = b->doms.size();
    for (mms_ctx *ctx : b->doms) {
        ctx->ctl_known = ctx->fs_part_valid = false;
        if ((st = read_ctl(ctx))) return st;
        if (ctx->h_ctl->status) return (mms_status)ctx->h_ctl->status;
        ctx->stepped = true;
    }
    if ((st = batch_refresh(b))) return st;
    std::vector<unsigned long long> ts0(nd);
    for (size_t i = 0; i < nd; i++) ts0[i] = b->doms[i]->h_ctl->timestep;
    const int chunk = 256;
    int done = 0;
    while (done < nsteps) {
        const int n = std::min(chunk, nsteps - done);
        if ((st = batch_ensure_graph(b))) return st;
        for (int s = 0; s < n; s++) {
            if (cudaGraphLaunch(b->graph, b->stream) != cudaSuccess) {
                b->err = "cudaGraphLaunch failed";
                return MMS_ERR_CUDA;
            }
            b->launches += b->graph_kernels;
        }
        // every domain's control block, one synchronisation
        for (mms_ctx *ctx : b->doms)
            cudaMemcpyAsync(ctx->h_ctl, ctx->ka.d.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, b->stream);
        if (cudaStreamSynchronize(b->stream) != cudaSuccess) {
            b->err = std::string("batch step: ") + cudaGetErrorString(cudaGetLastError());
            return MMS_ERR_CUDA;
        }
        done += n;
        for (size_t i = 0; i < nd; i++) {
            mms_ctx *ctx = b->doms[i];
            if (ctx->h_ctl->stall == STALL_ERROR) {
                b->err = "domain " + std::to_string(i) + ": " + mms_status_string((mms_status)ctx->h_ctl->status);
                return (mms_status)(ctx->h_ctl->status ? ctx->h_ctl->status : MMS_ERR_STATE);
            }
            if (ctx->h_ctl->stall == STALL_RNG && (st = batch_resume(ctx, ts0[i] + done))) {
                b->err = "domain " + std::to_string(i) + ": " + ctx->err;
                return st;
            }
            if ((st = refill_rng(ctx, false))) return st;
        }
    }
    return MMS_OK;
}

mms_status mms_batch_set_stencil_tile(mms_batch *b, int cells_per_thread, int zchunk)
{
    if (!b || (cells_per_thread != 1 && cells_per_thread != 2) || zchunk < 0 || zchunk > 64) return MMS_ERR_ARG;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    b->cpt = cells_per_thread;
    b->zc = zchunk;
    return batch_build_items(b);
}

mms_status mms_batch_get_stencil_tile(const mms_batch *b, int *cells_per_thread, int *zchunk, int *grid)
{
    if (!b) return MMS_ERR_ARG;
    if (cells_per_thread) *cells_per_thread = b->cpt;
    if (zchunk) *zchunk = b->zc;
    if (grid) *grid = b->grid;
    return MMS_OK;
}

// Batch tile autotuner: the persistent stencil over all domains is timed for
// every candidate tile on shadows of the fields it writes (as mms_autotune
// does for one domain); the fastest by median of `reps` launches is kept.
mms_status mms_batch_autotune(mms_batch *b, int reps, int *cells_per_thread, int *zchunk, double *best_ms)
{
    if (!b || reps < 1) return MMS_ERR_ARG;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    const size_t nd = b->doms.size();
    std::vector<void *> shadow;
    auto release = [&]() {
        cudaStreamSynchronize(b->stream);
        for (void *q : shadow) cudaFree(q);
    };
    std::vector<KernelArgs> sargs(nd);
    for (size_t i = 0; i < nd; i++) {
        mms_ctx *ctx = b->doms[i];
        mms_status st = read_ctl(ctx);
        if (st) {
            release();
            return st;
        }
        const Geo &g = ctx->ka.g;
        const size_t N = (size_t)g.N, rs = ctx->prec == MMS_PREC_F32 ? sizeof(float) : sizeof(double);
        KernelArgs sa = ctx->ka;
        const int pout = (int)((ctx->h_ctl->timestep + 1) & 1ULL);
        // es > 0: a field, placed as dalloc_field places it
        auto sh = [&](const void *src, size_t bytes, size_t es = 0) -> void * {
            void *raw = nullptr;
            if (cudaMalloc(&raw, bytes + (es ? 16 : 0)) != cudaSuccess) return nullptr;
            shadow.push_back(raw);
            void *d = es ? (void *)((char *)raw + 16 - es) : raw;
            cudaMemcpyAsync(d, src, bytes, cudaMemcpyDeviceToDevice, b->stream);
            return d;
        };
        sa.d.ce = sh(sa.d.ce, N * rs, rs);
        sa.d.cl[pout] = sh(sa.d.cl[pout], N * rs, rs);
        sa.d.fs[pout] = sh(sa.d.fs[pout], N * rs, rs);
        sa.d.gr = (int *)sh(sa.d.gr, N * sizeof(int), 4);
        sa.d.solid_bits = (unsigned *)sh(sa.d.solid_bits, (size_t)g.nwords * sizeof(unsigned));
        sa.d.ctl = (Ctl *)sh(sa.d.ctl, sizeof(Ctl));
        if (!sa.d.ce || !sa.d.cl[pout] || !sa.d.fs[pout] || !sa.d.gr || !sa.d.solid_bits || !sa.d.ctl) {
            release();
            b->err = "autotune shadow buffers: out of memory";
            return MMS_ERR_NOMEM;
        }
        Ctl c = *ctx->h_ctl;
        c.timestep += 1;
        c.status = 0;
        c.stall = 0;
        cudaMemcpyAsync(sa.d.ctl, &c, sizeof c, cudaMemcpyHostToDevice, b->stream);
        cudaStreamSynchronize(b->stream);
        sargs[i] = sa;
    }
    const size_t ib = batch_item_bytes();
    std::vector<unsigned char> host(ib * nd);
    void *ditems = nullptr;
    if (cudaMalloc(&ditems, host.size()) != cudaSuccess) {
        release();
        return MMS_ERR_NOMEM;
    }
    shadow.push_back(ditems);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 1e300;
    int bc = b->cpt, bz = b->zc;
    for (int cpt = 1; cpt <= 2; cpt++)
        for (int zc : {0, 8, 16, 32}) {
            long long tiles = 0;
            bool ok = true;
            for (size_t i = 0; i < nd && ok; i++) {
                TmaHolder th{};
                th.cpt = cpt;
                th.zc = zc;
                ok = make_tma(sargs[i], b->prec, th) != 0;
                tiles += fill_batch_item(host.data() + ib * i, sargs[i], th, tiles);
            }
            if (!ok) continue;
            cudaMemcpyAsync(ditems, host.data(), host.size(), cudaMemcpyHostToDevice, b->stream);
            cudaStreamSynchronize(b->stream);
            const int grid = batch_grid(b->prec, cpt);
            std::vector<float> ms;
            for (int r = 0; r < reps + 2; r++) {
                cudaEventRecord(e0, b->stream);
                launch_stencil_batch(ditems, (int)nd, tiles, b->prec, cpt, grid, b->stream);
                cudaEventRecord(e1, b->stream);
                cudaEventSynchronize(e1);
                float t = 0.f;
                cudaEventElapsedTime(&t, e0, e1);
                if (r >= 2) ms.push_back(t);
            }
            if (cudaGetLastError() != cudaSuccess) {
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                release();
                b->err = "batch autotune launch failed";
                return MMS_ERR_CUDA;
            }
            std::sort(ms.begin(), ms.end());
            if (ms[ms.size() / 2] < best) {
                best = ms[ms.size() / 2];
                bc = cpt;
                bz = zc;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    release();
    b->cpt = bc;
    b->zc = bz;
    mms_status st = batch_build_items(b);
    if (cells_per_thread) *cells_per_thread = bc;
    if (zchunk) *zchunk = bz;
    if (best_ms) *best_ms = best;
    return st;
}

uint64_t mms_batch_kernel_launches(const mms_batch *b) { return b ? b->launches : 0; }

const char *mms_batch_last_error(const mms_batch *b) { return b ? b->err.c_str() : ""; }

}  // extern "C"

// ================================================================ checkpoint
// Raw checkpoint of a context: every device array a later step reads (in
// the device layout), the control block, the grain table and log, the
// orientation tables, and the host side of the per-rank random streams
// (call counts, cached Gaussian, drawn orientations), the site list and the
// orientation overrides.  A context created from the same deck and loaded
// from it continues exactly as the saved one would have.
namespace {

struct CkHeader {
    char magic[8];
    int32_t version, prec, gx, gy, gz, nranks, rng_cap, num_grains;
    int64_t N, nsites, ninj, dctmp, P;
    uint64_t timestep;
};

bool fwrite_all(FILE *fp, const void *p, size_t n) { return n == 0 || std::fwrite(p, 1, n, fp) == n; }
bool fread_all(FILE *fp, void *p, size_t n) { return n == 0 || std::fread(p, 1, n, fp) == n; }

}  // namespace

extern "C" {

mms_status mms_checkpoint_save(mms_ctx *ctx, const char *path)
{
    Range range("mms_checkpoint_save");
    if (!ctx || !path) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    mms_status st = read_ctl(ctx);
    if (st) return st;
    const Geo &g = ctx->ka.g;
    const DevPtrs &d = ctx->ka.d;
    const size_t N = (size_t)g.N, es = ctx->prec == MMS_PREC_F32 ? sizeof(float) : sizeof(double);
    const Ctl c = *ctx->h_ctl;
    const int cur = (int)(c.timestep & 1ULL);
    CkHeader h{};
    std::memcpy(h.magic, "MMSCKPT", 8);
    h.version = 4;
    h.prec = ctx->prec;
    h.gx = g.gx;
    h.gy = g.gy;
    h.gz = g.gz;
    h.nranks = g.nranks;
    h.rng_cap = d.rng_cap;
    h.num_grains = c.num_grains;
    h.N = (int64_t)N;
    h.nsites = (int64_t)ctx->site_cell.size();
    h.ninj = (int64_t)ctx->inj_key.size();
    h.dctmp = (int64_t)g.nranks * (g.sbcells + 101);
    h.P = g.P;
    h.timestep = c.timestep;
    FILE *fp = std::fopen(path, "wb");
    if (!fp) return MMS_ERR_IO;
    std::vector<unsigned char> buf;
    bool ok = fwrite_all(fp, &h, sizeof h) && fwrite_all(fp, &c, sizeof c);
    auto dev = [&](const void *src, size_t bytes) {
        if (!ok) return;
        buf.resize(bytes);
        if (bytes && d2h(ctx, buf.data(), src, bytes) != cudaSuccess) ok = false;
        ok = ok && fwrite_all(fp, buf.data(), bytes);
    };
    dev(d.ce, N * es);
    dev(d.cl[cur], N * es);
    dev(d.fs[cur], N * es);
    dev(d.gr, N * sizeof(int));
    dev(d.dc, N * sizeof(Dc3));
    dev(d.dc_tmp, (size_t)h.dctmp * sizeof(Dc3));
    dev(d.rank_dcsize, (size_t)g.nranks * sizeof(int));
    dev(d.grain_rot, (size_t)c.num_grains * 9 * sizeof(double));
    dev(d.grain_log, (size_t)c.num_grains * sizeof(GrainLog));
    if (ctx->p.gnUseOrientation) {
        dev(d.rng_rot, (size_t)g.nranks * d.rng_cap * 9 * sizeof(double));
        dev(d.rng_used, (size_t)g.nranks * sizeof(int));
        dev(d.rng_base, (size_t)g.nranks * sizeof(long long));
    }
    if (d.lsindex) dev(d.lsindex, N * sizeof(int));
    for (const Rank &r : ctx->ranks) {
        const int64_t na = (int64_t)r.angles.size();
        ok = ok && fwrite_all(fp, &r.ncalls, sizeof r.ncalls) && fwrite_all(fp, &r.have_gauss, sizeof r.have_gauss) &&
             fwrite_all(fp, &r.gauss_next, sizeof r.gauss_next) && fwrite_all(fp, &r.rng_base, sizeof r.rng_base) &&
             fwrite_all(fp, &na, sizeof na) && fwrite_all(fp, r.angles.data(), (size_t)na * sizeof(r.angles[0]));
    }
    ok = ok && fwrite_all(fp, ctx->site_cell.data(), ctx->site_cell.size() * sizeof(long long)) &&
         fwrite_all(fp, ctx->site_thr.data(), ctx->site_thr.size() * sizeof(float)) &&
         fwrite_all(fp, ctx->site_rank.data(), ctx->site_rank.size() * sizeof(int)) &&
         fwrite_all(fp, ctx->inj_key.data(), ctx->inj_key.size() * sizeof(long long)) &&
         fwrite_all(fp, ctx->inj_rot.data(), ctx->inj_rot.size() * sizeof(double));
    {
        // XDMF state: rank 0's stream position before its undrawn
        // orientations (as a call count) and the last grain renumbering
        const int32_t sv = ctx->r0_snap_valid ? 1 : 0;
        const int64_t nr = (int64_t)ctx->renumber.size();
        ok = ok && fwrite_all(fp, &sv, sizeof sv) && fwrite_all(fp, &ctx->r0_snap_k, sizeof ctx->r0_snap_k) &&
             fwrite_all(fp, &ctx->r0_snap.ncalls, sizeof ctx->r0_snap.ncalls) &&
             fwrite_all(fp, &ctx->r0_snap.have_gauss, sizeof ctx->r0_snap.have_gauss) &&
             fwrite_all(fp, &ctx->r0_snap.gauss_next, sizeof ctx->r0_snap.gauss_next) && fwrite_all(fp, &nr, sizeof nr) &&
             fwrite_all(fp, ctx->renumber.data(), (size_t)nr * sizeof(uint64_t));
    }
    if (std::fclose(fp) != 0) ok = false;
    return ok ? MMS_OK : MMS_ERR_IO;
}

mms_status mms_checkpoint_load(mms_ctx *ctx, const char *path)
{
    Range range("mms_checkpoint_load");
    if (ctx) ctx->ctl_known = ctx->fs_part_valid = false;
    if (!ctx || !path) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    mms_status st = read_ctl(ctx);
    if (st) return st;
    const Geo &g = ctx->ka.g;
    DevPtrs &d = ctx->ka.d;
    const size_t N = (size_t)g.N, es = ctx->prec == MMS_PREC_F32 ? sizeof(float) : sizeof(double);
    FILE *fp = std::fopen(path, "rb");
    if (!fp) return MMS_ERR_IO;
    CkHeader h{};
    Ctl c{};
    auto fail = [&](mms_status s, const char *why) {
        std::fclose(fp);
        ctx->err = why;
        return s;
    };
    if (!fread_all(fp, &h, sizeof h) || std::memcmp(h.magic, "MMSCKPT", 8) != 0 || h.version != 4)
        return fail(MMS_ERR_IO, "not a checkpoint of this library");
    if (h.prec != ctx->prec || h.gx != g.gx || h.gy != g.gy || h.gz != g.gz || h.nranks != g.nranks ||
        h.rng_cap != d.rng_cap || h.N != (int64_t)N || h.P != g.P ||
        h.dctmp != (int64_t)g.nranks * (g.sbcells + 101) ||
        (uint64_t)h.num_grains > ctx->p.maxTotalGrains + 1)
        return fail(MMS_ERR_ARG, "checkpoint does not match this deck and form");
    if (!fread_all(fp, &c, sizeof c)) return fail(MMS_ERR_IO, "truncated checkpoint");
    const int cur = (int)(c.timestep & 1ULL);
    std::vector<unsigned char> buf;
    bool ok = true;
    auto dev = [&](void *dst, size_t bytes) {
        if (!ok) return;
        buf.resize(bytes);
        ok = fread_all(fp, buf.data(), bytes) && (bytes == 0 || h2d(ctx, dst, buf.data(), bytes) == cudaSuccess);
    };
    dev(d.ce, N * es);
    dev(d.cl[cur], N * es);
    dev(d.fs[cur], N * es);
    dev(d.gr, N * sizeof(int));
    dev(d.dc, N * sizeof(Dc3));
    dev(d.dc_tmp, (size_t)h.dctmp * sizeof(Dc3));
    dev(d.rank_dcsize, (size_t)g.nranks * sizeof(int));
    dev(d.grain_rot, (size_t)h.num_grains * 9 * sizeof(double));
    dev(d.grain_log, (size_t)h.num_grains * sizeof(GrainLog));
    if (ctx->p.gnUseOrientation) {
        dev(d.rng_rot, (size_t)g.nranks * d.rng_cap * 9 * sizeof(double));
        dev(d.rng_used, (size_t)g.nranks * sizeof(int));
        dev(d.rng_base, (size_t)g.nranks * sizeof(long long));
    }
    if (d.lsindex) dev(d.lsindex, N * sizeof(int));
    if (!ok) return fail(MMS_ERR_IO, "truncated checkpoint");
    for (Rank &r : ctx->ranks) {
        long ncalls = 0;
        int64_t na = 0;
        ok = ok && fread_all(fp, &ncalls, sizeof ncalls) && fread_all(fp, &r.have_gauss, sizeof r.have_gauss) &&
             fread_all(fp, &r.gauss_next, sizeof r.gauss_next) && fread_all(fp, &r.rng_base, sizeof r.rng_base) &&
             fread_all(fp, &na, sizeof na);
        if (!ok || na < 0) return fail(MMS_ERR_IO, "truncated checkpoint");
        r.angles.resize((size_t)na);
        ok = fread_all(fp, r.angles.data(), (size_t)na * sizeof(r.angles[0]));
        // the random_r state: reseed and replay the same number of calls
        const int hg = r.have_gauss;
        const float gn = r.gauss_next;
        r.seed_with(r.seed);
        while (r.ncalls < ncalls) r.rand_();
        r.have_gauss = hg;
        r.gauss_next = gn;
    }
    ctx->site_cell.resize((size_t)h.nsites);
    ctx->site_thr.resize((size_t)h.nsites);
    ctx->site_rank.resize((size_t)h.nsites);
    ctx->inj_key.resize((size_t)h.ninj);
    ctx->inj_rot.resize((size_t)h.ninj * 9);
    ok = ok && fread_all(fp, ctx->site_cell.data(), ctx->site_cell.size() * sizeof(long long)) &&
         fread_all(fp, ctx->site_thr.data(), ctx->site_thr.size() * sizeof(float)) &&
         fread_all(fp, ctx->site_rank.data(), ctx->site_rank.size() * sizeof(int)) &&
         fread_all(fp, ctx->inj_key.data(), ctx->inj_key.size() * sizeof(long long)) &&
         fread_all(fp, ctx->inj_rot.data(), ctx->inj_rot.size() * sizeof(double));
    {
        int32_t sv = 0;
        int64_t nr = 0;
        long snap_calls = 0;
        int hg = 0;
        float gn = 0.f;
        ok = ok && fread_all(fp, &sv, sizeof sv) && fread_all(fp, &ctx->r0_snap_k, sizeof ctx->r0_snap_k) &&
             fread_all(fp, &snap_calls, sizeof snap_calls) && fread_all(fp, &hg, sizeof hg) &&
             fread_all(fp, &gn, sizeof gn) && fread_all(fp, &nr, sizeof nr) && nr >= 0;
        if (ok) {
            ctx->renumber.resize((size_t)nr);
            ok = fread_all(fp, ctx->renumber.data(), (size_t)nr * sizeof(uint64_t));
        }
        ctx->r0_snap_valid = ok && sv && !ctx->ranks.empty();
        if (ctx->r0_snap_valid) {
            // the stream position by replay from the seed
            Rank tmp;
            tmp.seed_with(ctx->ranks[0].seed);
            while (tmp.ncalls < snap_calls) tmp.rand_();
            tmp.have_gauss = hg;
            tmp.gauss_next = gn;
            tmp.save(ctx->r0_snap);
        }
    }
    std::fclose(fp);
    if (!ok) {
        ctx->err = "truncated checkpoint";
        return MMS_ERR_IO;
    }
    ctx->site_index.clear();
    if ((st = upload_sites(ctx))) return st;
    dfree(ctx, d.inj_key);
    dfree(ctx, d.inj_rot);
    d.inj_key = nullptr;
    d.inj_rot = nullptr;
    d.n_inj = (long long)ctx->inj_key.size();
    if (d.n_inj) {
        if ((st = dalloc(ctx, &d.inj_key, (size_t)d.n_inj)) || (st = dalloc(ctx, &d.inj_rot, 9 * (size_t)d.n_inj)))
            return st;
        CU(h2d(ctx, d.inj_key, ctx->inj_key.data(), (size_t)d.n_inj * sizeof(long long)));
        CU(h2d(ctx, d.inj_rot, ctx->inj_rot.data(), 9 * (size_t)d.n_inj * sizeof(double)));
    }
    c.status = 0;
    c.stall = 0;
    CU(h2d(ctx, d.ctl, &c, sizeof c));
    *ctx->h_ctl = c;
    ctx->grains.assign(1, mms_grain{});
    ctx->grains_synced = 1;
    ctx->stepped = true;
    drop_graph(ctx);
    return MMS_OK;
}

}  // extern "C"

// ============================================== z-slab split of one domain
// The reference splits its domain into NSubblocks MPI ranks that exchange
// halo planes and grain lists inside doiteration (calculate.c:193-352).
// Here the split is into z-slabs of whole subblock layers, one context per
// slab: the emulated ranks, their streams, interface lists and dc_tmp
// slots stay inside one slab, and a step needs two exchanges:
//   point 0, after nucleation: the cl and fs boundary planes of the step's
//     input buffers, and every slab's {candidates, short of draws};
//   point 1, after the stencil: the fs (output buffer), gr, dc and solid
//     bitmask boundary planes, and every slab's new grains.
namespace {

// Transfers of one exchange point for the step that starts at timestep ts
// (its input buffers are ts & 1).  Halo entries come per neighbour in a
// fixed field order, so a slab's entries for peer q and q's entries for
// this slab pair up one to one.
void slab_plan(mms_ctx *ctx, int point, unsigned long long ts, std::vector<mms_slab_xfer> &out)
{
    out.clear();
    const Geo &g = ctx->ka.g;
    const DevPtrs &d = ctx->ka.d;
    const size_t es = elem_size(ctx);
    const int bin = (int)(ts & 1ULL), bout = (int)((ts + 1) & 1ULL);
    struct Field {
        void *base;
        size_t plane;  // bytes of one z-plane
    };
    std::vector<Field> f;
    if (point == 0) {
        f.push_back({d.cl[bin], (size_t)g.sz * es});
        f.push_back({d.fs[bin], (size_t)g.sz * es});
    } else {
        f.push_back({d.fs[bout], (size_t)g.sz * es});
        f.push_back({d.gr, (size_t)g.sz * sizeof(int)});
        f.push_back({d.dc, (size_t)g.sz * sizeof(Dc3)});
        f.push_back({d.solid_bits, (size_t)g.wpr * (g.gy + 2) * sizeof(unsigned)});
    }
    auto plane = [](const Field &x, long long k) { return (void *)((char *)x.base + (size_t)k * x.plane); };
    if (ctx->slab > 0)
        for (const Field &x : f) out.push_back({MMS_XFER_HALO, ctx->slab - 1, plane(x, 1), plane(x, 0), x.plane});
    if (ctx->slab < ctx->nslabs - 1)
        for (const Field &x : f)
            out.push_back({MMS_XFER_HALO, ctx->slab + 1, plane(x, g.gz), plane(x, g.gz + 1), x.plane});
    if (point == 0) out.push_back({MMS_XFER_GATHER, -1, d.x1_send, d.x1_recv, 2 * sizeof(int)});
    else out.push_back({MMS_XFER_GATHER, -1, d.x2_send, d.x2_recv, (uint64_t)d.slab_cap * sizeof(SlabRow)});
}

mms_status slab_launch(mms_ctx *ctx, int phase, int resume)
{
    cudaSetDevice(ctx->device);
    ctx->ctl_known = ctx->fs_part_valid = false;
    if (phase == 0 && !resume && ctx->p.am)
        ctx->launches += launch_temp_am(ctx->ka, am_params(ctx->p), ctx->prec, ctx->stream, nullptr, ctx->am_rows);
    ctx->launches += launch_slab_phase(ctx->ka, ctx->tma, ctx->prec, ctx->stream, phase, resume);
    CU(cudaGetLastError());
    return MMS_OK;
}

// Slab b pulls what point `point` brings it, on its own stream, after the
// phase each source slab recorded in ev[source].
mms_status slab_pull(mms_ctx *const *slabs, int S, int b, int point, unsigned long long ts, int ev)
{
    mms_ctx *ctx = slabs[b];
    std::vector<mms_slab_xfer> mine, theirs;
    slab_plan(ctx, point, ts, mine);
    cudaSetDevice(ctx->device);
    auto copy = [&](void *dst, const mms_ctx *src_ctx, const void *src, size_t bytes) -> cudaError_t {
        cudaError_t e = cudaStreamWaitEvent(ctx->stream, src_ctx->slab_events[ev], 0);
        if (e != cudaSuccess) return e;
        if (src_ctx->device == ctx->device)
            return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, ctx->stream);
        return cudaMemcpyPeerAsync(dst, ctx->device, src, src_ctx->device, bytes, ctx->stream);
    };
    for (int peer : {b - 1, b + 1}) {
        if (peer < 0 || peer >= S) continue;
        slab_plan(slabs[peer], point, ts, theirs);
        std::vector<const mms_slab_xfer *> a, q;
        for (const mms_slab_xfer &x : mine)
            if (x.kind == MMS_XFER_HALO && x.peer == peer) a.push_back(&x);
        for (const mms_slab_xfer &x : theirs)
            if (x.kind == MMS_XFER_HALO && x.peer == b) q.push_back(&x);
        if (a.size() != q.size()) {
            ctx->err = "slab exchange plans do not pair";
            return MMS_ERR_STATE;
        }
        for (size_t i = 0; i < a.size(); i++) CU(copy(a[i]->recv, slabs[peer], q[i]->send, a[i]->bytes));
    }
    const mms_slab_xfer *gm = nullptr;
    for (const mms_slab_xfer &x : mine)
        if (x.kind == MMS_XFER_GATHER) gm = &x;
    for (int a = 0; a < S; a++) {
        slab_plan(slabs[a], point, ts, theirs);
        for (const mms_slab_xfer &x : theirs)
            if (x.kind == MMS_XFER_GATHER) {
                if (x.bytes != gm->bytes) {
                    ctx->err = "slab gather sizes differ";
                    return MMS_ERR_STATE;
                }
                CU(copy((char *)gm->recv + (size_t)a * gm->bytes, slabs[a], x.send, x.bytes));
            }
    }
    return MMS_OK;
}

// One step of every slab (resume: the step that stalled at activation).
// Events per slab: 0 after phase 0, 1 after phase 1, 2 after its pulls of
// point 1; phase 2 of every slab waits for every slab's pulls, since they
// read its planes and rows.
mms_status slab_group_one(mms_ctx *const *slabs, int S, unsigned long long ts, int resume)
{
    mms_status st;
    auto record = [&](int s, int ev) -> mms_status {
        mms_ctx *ctx = slabs[s];
        cudaSetDevice(ctx->device);
        CU(cudaEventRecord(ctx->slab_events[ev], ctx->stream));
        return MMS_OK;
    };
    for (int s = 0; s < S; s++)
        if ((st = slab_launch(slabs[s], 0, resume)) || (st = record(s, 0))) return st;
    for (int s = 0; s < S; s++)
        if ((st = slab_pull(slabs, S, s, 0, ts, 0))) return st;
    for (int s = 0; s < S; s++)
        if ((st = slab_launch(slabs[s], 1, 0)) || (st = record(s, 1))) return st;
    for (int s = 0; s < S; s++)
        if ((st = slab_pull(slabs, S, s, 1, ts, 1)) || (st = record(s, 2))) return st;
    for (int s = 0; s < S; s++) {
        mms_ctx *ctx = slabs[s];
        cudaSetDevice(ctx->device);
        for (int q = 0; q < S; q++)
            if (q != s) CU(cudaStreamWaitEvent(ctx->stream, slabs[q]->slab_events[2], 0));
        if ((st = slab_launch(ctx, 2, 0))) return st;
    }
    return MMS_OK;
}

}  // namespace

extern "C" {

mms_status mms_slab_layout_of(const mms_params *global, int nslabs, int slab, mms_slab_layout *out)
{
    if (!global || !out) return MMS_ERR_ARG;
    int L0, L1;
    if (global->gnsbz < 1 || !slab_span(*global, nslabs, slab, L0, L1)) return MMS_ERR_ARG;
    out->nslabs = nslabs;
    out->slab = slab;
    out->z_begin = L0 * global->gsdimz;
    out->z_cells = (L1 - L0) * global->gsdimz;
    out->rank_begin = L0 * global->gnsbx * global->gnsby;
    out->rank_count = (L1 - L0) * global->gnsbx * global->gnsby;
    return MMS_OK;
}

mms_status mms_slab_get_layout(const mms_ctx *ctx, mms_slab_layout *out)
{
    if (!ctx) return MMS_ERR_ARG;
    return mms_slab_layout_of(&ctx->gp, ctx->nslabs, ctx->slab, out);
}

mms_status mms_slab_launch(mms_ctx *ctx, int phase, int resume)
{
    if (!ctx || phase < 0 || phase > 2 || (resume && phase != 0)) return MMS_ERR_ARG;
    ctx->stepped = true;
    return slab_launch(ctx, phase, resume);
}

mms_status mms_slab_exchange_plan(mms_ctx *ctx, int point, uint64_t timestep, mms_slab_xfer *out, int max, int *n)
{
    if (!ctx || !n || point < 0 || point > 1 || max < 0 || (max && !out)) return MMS_ERR_ARG;
    if (ctx->nslabs < 2) {
        *n = 0;
        return MMS_OK;
    }
    std::vector<mms_slab_xfer> v;
    slab_plan(ctx, point, timestep, v);
    *n = (int)v.size();
    if ((int)v.size() > max) return MMS_ERR_ARG;
    std::copy(v.begin(), v.end(), out);
    return MMS_OK;
}

mms_status mms_slab_poll(mms_ctx *ctx, uint64_t *timestep, int *stalled)
{
    if (!ctx) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    mms_status st = read_ctl(ctx);
    if (st) return st;
    const Ctl &c = *ctx->h_ctl;
    if (c.stall == STALL_ERROR) return (mms_status)(c.status ? c.status : MMS_ERR_STATE);
    if (timestep) *timestep = c.timestep;
    if (stalled) *stalled = (c.stall == STALL_RNG) ? 1 : 0;
    return MMS_OK;
}

mms_status mms_slab_refill(mms_ctx *ctx)
{
    if (!ctx) return MMS_ERR_ARG;
    ctx->ctl_known = ctx->fs_part_valid = false;
    cudaSetDevice(ctx->device);
    mms_status st = read_ctl(ctx);
    if (st) return st;
    if ((st = refill_rng(ctx, ctx->h_ctl->stall == STALL_RNG))) return st;
    if (ctx->h_ctl->stall == STALL_RNG) {
        int zero = 0;
        CU(h2d(ctx, &ctx->ka.d.ctl->stall, &zero, sizeof(int)));
    }
    return MMS_OK;
}

mms_status mms_slab_group_step(mms_ctx *const *slabs, int nslabs, int nsteps)
{
    Range range("mms_slab_group_step");
    if (!slabs || nslabs < 1 || nsteps < 0) return MMS_ERR_ARG;
    for (int s = 0; s < nslabs; s++) {
        mms_ctx *c = slabs[s];
        if (!c || c->nslabs != nslabs || c->slab != s || c->prec != slabs[0]->prec ||
            c->gg.N != slabs[0]->gg.N || c->ka.d.slab_cap != slabs[0]->ka.d.slab_cap)
            return MMS_ERR_ARG;
    }
    if (nslabs == 1) return mms_step(slabs[0], nsteps);
    mms_status st;
    for (int s = 0; s < nslabs; s++) {
        mms_ctx *c = slabs[s];
        c->stepped = true;
        cudaSetDevice(c->device);
        while (c->slab_events.size() < 3) {
            cudaEvent_t e;
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
                c->err = "cudaEventCreateWithFlags failed";
                return MMS_ERR_CUDA;
            }
            c->slab_events.push_back(e);
        }
        for (int q = 0; q < nslabs; q++)
            if (slabs[q]->device != c->device) {
                cudaError_t e = cudaDeviceEnablePeerAccess(slabs[q]->device, 0);
                if (e != cudaSuccess) cudaGetLastError();  // already enabled, or copies are staged
            }
    }
    // every slab at the same step, none stalled
    uint64_t ts = 0;
    for (int s = 0; s < nslabs; s++) {
        uint64_t t;
        int stl;
        if ((st = mms_slab_poll(slabs[s], &t, &stl))) return st;
        if (s == 0) ts = t;
        if (t != ts || stl) {
            slabs[s]->err = "slabs are not at the same step";
            return MMS_ERR_STATE;
        }
    }
    const uint64_t target = ts + (uint64_t)nsteps;
    const int chunk = 256;
    while (ts < target) {
        const int n = (int)std::min<uint64_t>(chunk, target - ts);
        for (int k = 0; k < n; k++)
            if ((st = slab_group_one(slabs, nslabs, ts + k, 0))) return st;
        // a stall stops every slab at the same activation, and the steps
        // launched after it do nothing (their exchanges copy unchanged data)
        int stl = 0;
        uint64_t t = 0;
        for (int s = 0; s < nslabs; s++) {
            int x;
            uint64_t ts_s;
            if ((st = mms_slab_poll(slabs[s], &ts_s, &x))) return st;
            if (s == 0) t = ts_s, stl = x;
            if (ts_s != t || x != stl) {
                slabs[s]->err = "slabs diverged";
                return MMS_ERR_STATE;
            }
        }
        if (stl) {
            for (int s = 0; s < nslabs; s++)
                if ((st = mms_slab_refill(slabs[s]))) return st;
            if ((st = slab_group_one(slabs, nslabs, t, 1))) return st;
            ts = t + 1;
            continue;  // poll again before going on
        }
        ts = t;
        for (int s = 0; s < nslabs; s++)
            if ((st = refill_rng(slabs[s], false))) return st;
    }
    return MMS_OK;
}

// ---- one process per device over NCCL -----------------------------------

mms_status mms_slab_nccl_unique_id(const char *nccl_path, void *id128)
{
    if (!id128) return MMS_ERR_ARG;
    const NcclApi *n = nccl_api(nccl_path, nullptr);
    if (!n) return MMS_ERR_ARG;
    ncclUniqueId id;
    if (n->GetUniqueId(&id) != ncclSuccess) return MMS_ERR_CUDA;
    std::memcpy(id128, &id, sizeof id);
    return MMS_OK;
}

mms_status mms_slab_nccl_init(mms_ctx *ctx, const char *nccl_path, const void *id128)
{
    if (!ctx || !id128) return MMS_ERR_ARG;
    if (ctx->nccl_comm) return MMS_ERR_STATE;
    std::string err;
    const NcclApi *n = nccl_api(nccl_path, &err);
    if (!n) {
        ctx->err = err;
        return MMS_ERR_ARG;
    }
    cudaSetDevice(ctx->device);
    if (!ctx->nccl_scratch) {
        long long *p = nullptr;
        mms_status st = dalloc(ctx, &p, 8);
        if (st) return st;
        ctx->nccl_scratch = p;
    }
    ncclUniqueId id;
    std::memcpy(&id, id128, sizeof id);
    ncclComm_t comm = nullptr;
    const ncclResult_t r = n->CommInitRank(&comm, ctx->nslabs, id, ctx->slab);
    if (r != ncclSuccess) {
        ctx->err = std::string("ncclCommInitRank: ") + n->GetErrorString(r);
        return MMS_ERR_CUDA;
    }
    ctx->nccl_comm = comm;
    return MMS_OK;
}

}  // extern "C"

namespace {

mms_status nccl_fail(mms_ctx *ctx, const char *what, ncclResult_t r)
{
    ctx->err = std::string(what) + ": " + g_nccl.GetErrorString(r);
    return MMS_ERR_CUDA;
}

// One exchange point of the plan (slab_plan), as one NCCL group on the
// slab's stream: the halo planes as send/recv pairs with the neighbouring
// slabs, the gather as an all-gather.
mms_status nccl_exchange(mms_ctx *ctx, int point, unsigned long long ts)
{
    std::vector<mms_slab_xfer> v;
    slab_plan(ctx, point, ts, v);
    for (const mms_slab_xfer &x : v)
        if (!x.send || !x.recv) {  // a slab context without its exchange buffers
            ctx->err = "slab exchange buffers missing";
            return MMS_ERR_STATE;
        }
    ncclComm_t comm = (ncclComm_t)ctx->nccl_comm;
    ncclResult_t r = g_nccl.GroupStart();
    for (const mms_slab_xfer &x : v) {
        if (r != ncclSuccess) break;
        if (x.kind == MMS_XFER_HALO) {
            r = g_nccl.Send(x.send, (size_t)x.bytes, ncclUint8, x.peer, comm, ctx->stream);
            if (r == ncclSuccess) r = g_nccl.Recv(x.recv, (size_t)x.bytes, ncclUint8, x.peer, comm, ctx->stream);
        } else {
            r = g_nccl.AllGather(x.send, x.recv, (size_t)x.bytes, ncclUint8, comm, ctx->stream);
        }
    }
    const ncclResult_t r2 = g_nccl.GroupEnd();
    if (r != ncclSuccess) return nccl_fail(ctx, "NCCL exchange", r);
    if (r2 != ncclSuccess) return nccl_fail(ctx, "ncclGroupEnd", r2);
    return MMS_OK;
}

mms_status nccl_one(mms_ctx *ctx, unsigned long long ts, int resume)
{
    mms_status st;
    if ((st = slab_launch(ctx, 0, resume)) || (st = nccl_exchange(ctx, 0, ts)) || (st = slab_launch(ctx, 1, 0)) ||
        (st = nccl_exchange(ctx, 1, ts)) || (st = slab_launch(ctx, 2, 0)))
        return st;
    return MMS_OK;
}

// This slab's {timestep, stalled for orientations, error status}, and
// whether every slab of the group holds the same triple (an all-reduce of
// the values and their negatives with MAX); v[2] becomes the group's
// largest error status.
mms_status nccl_agree(mms_ctx *ctx, long long v[3], bool *same)
{
    mms_status st = read_ctl(ctx);
    if (st) return st;
    const Ctl &c = *ctx->h_ctl;
    v[0] = (long long)c.timestep;
    v[1] = c.stall == STALL_RNG ? 1 : 0;
    v[2] = c.stall == STALL_ERROR ? (c.status ? c.status : MMS_ERR_STATE) : 0;
    long long h[6] = {v[0], v[1], v[2], -v[0], -v[1], -v[2]};
    long long *d = (long long *)ctx->nccl_scratch;
    CU(cudaMemcpyAsync(d, h, sizeof h, cudaMemcpyHostToDevice, ctx->stream));
    const ncclResult_t r = g_nccl.AllReduce(d, d, 6, ncclInt64, ncclMax, (ncclComm_t)ctx->nccl_comm, ctx->stream);
    if (r != ncclSuccess) return nccl_fail(ctx, "ncclAllReduce", r);
    CU(cudaMemcpyAsync(h, d, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    *same = h[0] == -h[3] && h[1] == -h[4] && h[2] == -h[5];
    v[2] = h[2];
    return MMS_OK;
}

}  // namespace

extern "C" {

mms_status mms_slab_nccl_step(mms_ctx *ctx, int nsteps)
{
    Range range("mms_slab_nccl_step");
    if (!ctx || nsteps < 0) return MMS_ERR_ARG;
    if (!ctx->nccl_comm) return MMS_ERR_STATE;
    cudaSetDevice(ctx->device);
    ctx->stepped = true;
    long long v[3];
    bool same = false;
    mms_status st;
    if ((st = nccl_agree(ctx, v, &same))) return st;
    if (!same) {
        ctx->err = "slabs are not at the same step";
        return MMS_ERR_STATE;
    }
    if (v[2]) return (mms_status)v[2];
    if (v[1]) {
        ctx->err = "slab is stalled before stepping";
        return MMS_ERR_STATE;
    }
    // a group of one slab has nothing to exchange: its context steps like a
    // whole domain (as mms_slab_group_step does; its exchange buffers are
    // not allocated), and the group only checks that it agrees
    if (ctx->nslabs == 1) {
        if ((st = mms_step(ctx, nsteps)) || (st = nccl_agree(ctx, v, &same))) return st;
        if (!same) {
            ctx->err = "slabs diverged (timestep or stall state differs between ranks)";
            return MMS_ERR_STATE;
        }
        return v[2] ? (mms_status)v[2] : MMS_OK;
    }
    unsigned long long ts = (unsigned long long)v[0];
    const unsigned long long target = ts + (unsigned long long)nsteps;
    const int chunk = 64;
    while (ts < target) {
        const int n = (int)std::min<unsigned long long>(chunk, target - ts);
        for (int k = 0; k < n; k++)
            if ((st = nccl_one(ctx, ts + k, 0))) return st;
        // every slab reaches the same state: the same step, and a stall
        // (a shortage of pre-drawn orientations anywhere) at the same
        // activation, after which the launched steps did nothing
        if ((st = nccl_agree(ctx, v, &same))) return st;
        if (!same) {
            ctx->err = "slabs diverged (timestep or stall state differs between ranks)";
            return MMS_ERR_STATE;
        }
        if (v[2]) return (mms_status)v[2];
        if (v[1]) {
            if ((st = mms_slab_refill(ctx)) || (st = nccl_one(ctx, (unsigned long long)v[0], 1))) return st;
            ts = (unsigned long long)v[0] + 1;
            continue;
        }
        ts = (unsigned long long)v[0];
        if ((st = refill_rng(ctx, false))) return st;
    }
    return MMS_OK;
}

mms_status mms_slab_nccl_reduce(mms_ctx *ctx, mms_reduction what, double *out)
{
    if (!ctx || !out) return MMS_ERR_ARG;
    if (!ctx->nccl_comm) return MMS_ERR_STATE;
    const bool frac = what == MMS_REDUCE_FS_FRACTION;
    double local = 0.0;
    mms_status st = mms_reduce(ctx, frac ? MMS_REDUCE_SOLID_VOLUME : what, &local);
    if (st) return st;
    cudaSetDevice(ctx->device);
    double *d = (double *)ctx->nccl_scratch;
    CU(cudaMemcpyAsync(d, &local, sizeof local, cudaMemcpyHostToDevice, ctx->stream));
    const ncclResult_t r = g_nccl.AllReduce(d, d, 1, ncclFloat64, ncclSum, (ncclComm_t)ctx->nccl_comm, ctx->stream);
    if (r != ncclSuccess) return nccl_fail(ctx, "ncclAllReduce", r);
    double sum = 0.0;
    CU(cudaMemcpyAsync(&sum, d, sizeof sum, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    if (frac) {
        const mms_params &g = ctx->gp;
        const double cells = (double)((long long)g.gnsbx * g.gsdimx * (long long)g.gnsby * g.gsdimy *
                                      (long long)g.gnsbz * g.gsdimz);
        sum = sum / (cells * std::pow(g.cellSize, 3.0));
    }
    *out = sum;
    return MMS_OK;
}

}  // extern "C"

// ===================================================================== XDMF
namespace {

// getRenumberArray (io_xdmf.c:344-375): when the grain count has grown since
// the last renumbering, a fresh shuffle of the ids 1..n-1 drawn from rank
// 0's rand() stream.  Those draws come at the point the run has reached on
// that stream: after its setup draws and the orientation draws consumed so
// far.  Rank 0's later orientations therefore follow them, so its
// pre-drawn orientation table is redrawn from there.
mms_status xdmf_renumber(mms_ctx *ctx)
{
    const int ng = ctx->h_ctl->num_grains;
    if (!ctx->renumber.empty() && (size_t)ng <= ctx->renumber.size()) return MMS_OK;
    Rank &r = ctx->ranks[0];
    const DevPtrs &d = ctx->ka.d;
    long long k = 0;  // orientation draws rank 0 has consumed
    if (ctx->p.gnUseOrientation && d.rng_used) {
        int used0 = 0;
        CU(d2h(ctx, &used0, d.rng_used, sizeof(int)));
        k = r.rng_base + used0;
    }
    if (ctx->r0_snap_valid) {
        r.restore(ctx->r0_snap);
        for (long long i = ctx->r0_snap_k; i < k; i++) {
            NucPt n{};
            draw_orientation(ctx->p, r, n);
        }
    } else if (k != 0) {
        ctx->err = "rank 0's stream position is unknown";
        return MMS_ERR_STATE;
    }
    std::vector<uint64_t> a((size_t)ng);
    for (int i = 0; i < ng; i++) a[i] = (uint64_t)i;
    for (int i = 1; i < ng; i++) {
        int pic;
        do {
            pic = r.rand_() % ng;
        } while (pic == 0);
        std::swap(a[pic], a[i]);
    }
    ctx->renumber.swap(a);
    r.save(ctx->r0_snap);
    ctx->r0_snap_k = k;
    ctx->r0_snap_valid = true;
    if (ctx->p.gnUseOrientation && d.rng_used) {
        r.angles.resize((size_t)k);
        return refill_rng(ctx, true);
    }
    return MMS_OK;
}

}  // namespace

extern "C" {

mms_status mms_write_xdmf(mms_ctx *ctx, const char *basename)
{
    Range range("mms_write_xdmf");
    if (!ctx || ctx->nslabs > 1) return MMS_ERR_ARG;
    cudaSetDevice(ctx->device);
    const mms_params &p = ctx->p;
    const size_t n = (size_t)ctx->ka.g.rN;
    std::vector<double> T(n), ce(n), fs(n);
    std::vector<int32_t> gr(n);
    mms_status st;
    if ((st = mms_download(ctx, MMS_FIELD_TEMPERATURE, T.data())) || (st = mms_download(ctx, MMS_FIELD_CE, ce.data())) ||
        (st = mms_download(ctx, MMS_FIELD_GR, gr.data())) || (st = mms_download(ctx, MMS_FIELD_FS, fs.data())) ||
        (st = sync_grains(ctx)))
        return st;
    const int ng = ctx->h_ctl->num_grains;
    std::vector<double> ang((size_t)ng * 3);
    for (int i = 0; i < ng; i++)
        for (int a = 0; a < 3; a++) ang[3 * (size_t)i + a] = ctx->grains[i].rotang[a];
    if (p.randomize_grains && (st = xdmf_renumber(ctx))) return st;
    const std::string base = basename ? basename : p.basefilename;
    const int64_t ts = (int64_t)ctx->h_ctl->timestep;
    if (base != ctx->xdmf_base) {
        ctx->xdmf_base = base;
        ctx->xdmf_series.clear();
    }
    if (ctx->xdmf_series.empty() || ctx->xdmf_series.back() != ts) ctx->xdmf_series.push_back(ts);
    return mms_write_xdmf_arrays(&p, base.c_str(), ctx->xdmf_series.data(), (int)ctx->xdmf_series.size(), T.data(),
                                 ce.data(), gr.data(), fs.data(), ng, ang.data(),
                                 p.randomize_grains ? ctx->renumber.data() : nullptr);
}

mms_status mms_xdmf_renumbering(mms_ctx *ctx, int capacity, uint64_t *out, int *count)
{
    if (!ctx || !count || capacity < 0 || (capacity && !out)) return MMS_ERR_ARG;
    *count = (int)ctx->renumber.size();
    std::copy(ctx->renumber.begin(), ctx->renumber.begin() + std::min<size_t>(ctx->renumber.size(), (size_t)capacity),
              out);
    return MMS_OK;
}

}  // extern "C"
