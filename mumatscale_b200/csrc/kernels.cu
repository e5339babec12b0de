// kernels.cu — sm_100a kernels for one muMatScale CA timestep.
//
// Compiled with -fmad=false: every FP64 expression is evaluated with the
// same rounding, in the same order, as the reference's gcc x86-64 build
// (which contracts nothing), so the FP64 plain form is bit-identical to it.
//
// One step (doiteration, calculate.c:193-352) is this launch sequence on one
// stream; every kernel reads the step number from the device control block,
// so the sequence can be replayed (or graph-captured) without the host:
//
//   k_temp_am     AM quadrature temperature (temperature.c:62-123), AM only
//   k_nuc         nucleation test over the pre-drawn sites (grain.c:1222-1285)
//   k_act         ordered grain activation (grain.c:840-916, 347-425)
//   k_curv        Gibbs-Thomson curvature (curvature.c:31-405), TipCurvature only
//   k_diffuse_fs  diffusion + fs change fused (growth.c:30-170, 177-276); also
//                 writes the solid-cell bitmask (gr > 0 after fs change)
//   k_list        interface list in rank-local raster order, membership from
//                 the bitmask (growth.c:461-538), in one pass (decoupled
//                 look-back); per-rank dc_tmp bookkeeping (growth.c:642-660)
//   k_capture     octahedron capture over the list (growth.c:339-407, 664-794),
//                 dc copy-back and captured grain ids (growth.c:789, 797-807)
//
// Fields: ce in place; cl and fs ping-pong between two buffers, the state
// after step t living in buffer (t & 1).  gr, dc in place.  d is never
// stored: capture recomputes it from the solid neighbour's dc, fs and
// grain rotation, which is exactly what grow_octahedra stored for it.
// Arrays use the device layout of Geo (row pitch P).
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <type_traits>

#include "device_common.cuh"
#include "mms_internal.h"

namespace mms {

#define FULL_MASK 0xffffffffu



template <int NT>
__device__ __forceinline__ int block_exclusive_scan(int v, int &total, int *sh)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(FULL_MASK, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = (lane < NT / 32) ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(FULL_MASK, w, o);
            if (lane >= o) w += y;
        }
        if (lane < NT / 32) sh[lane] = w;
    }
    __syncthreads();
    int prefix = warp ? sh[warp - 1] : 0;
    total = sh[NT / 32 - 1];
    __syncthreads();
    return prefix + x - v;
}

template <int NT>
__device__ __forceinline__ int block_sum(int v, int *sh)
{
    int t;
    block_exclusive_scan<NT>(v, t, sh);
    return t;
}

// ------------------------------------------------------- mbarrier + TMA
__device__ __forceinline__ unsigned smem_u32(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: gives up after 2^22 polls (about a second).  try_wait
// itself suspends the thread until the phase completes or a hardware time
// limit passes, so the first 2^14 polls follow each other directly; only a
// long wait backs off with short sleeps (a longer sleep delays the wake-up
// of every warp waiting on a plane that has just landed).
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity)
{
    for (unsigned it = 0; it < (1u << 22); it++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (it > (1u << 14)) __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                            unsigned long long *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"((unsigned long long)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// ------------------------------------------------------------ temperature
// AM moving-source quadrature, direct_temp_calc thermal_ana == 1
// (temperature.c:62-123), for step ctl->timestep + 1 over every halo'd cell:
//   T = liniT + Tfront sum_i ldt exp(-((lx + v t_i)^2 + ly^2)/a_i - lz^2/b_i) / Tl_i
// with a_i = s^2 + 4 alpha t_i, b_i = 4 alpha t_i, 400 midpoint nodes t_i.
// The exponential of the sum is the product of one factor per axis, so the
// sum is a contraction over i of three tables, X_i(x), Y_i(y) and
// Z_i(z) = ldt exp(-lz^2/b_i) / Tl_i, built once per step (k_am_tables),
// instead of 400 exponentials per cell (k_am_contract).  Cells above the
// substrate top (rz > znow + dx) get T = 0.
// tables: X [AM_NT][gx+2], Y [AM_NT][gy+2], Z [AM_NT][gz+2], then the
// per-plane flag "below the substrate top" [gz+2]
template <typename Real>
__global__ void k_am_tables(KernelArgs a, AmParams m)
{
    const Ctl *ctl = a.d.ctl;
    if (stalled(ctl)) return;
    const Geo &g = a.g;
    const Phys &p = a.p;
    // the step's source position and constants, formed once per CTA
    __shared__ AmStep s_step;
    if (threadIdx.x == 0) s_step = am_step(p, m, ctl->timestep + 1);
    __syncthreads();
    const AmStep s = s_step;
    const int nx = g.gx + 2, ny = g.gy + 2, nz = g.gz + 2, nc = nx + ny + nz;
    Real *X = (Real *)a.d.am_tab, *Y = X + (long long)AM_NT * nx, *Z = Y + (long long)AM_NT * ny;
    int *zon = (int *)(Z + (long long)AM_NT * nz);
    // fewer than 2^31 table entries (400 per halo'd row or column): 32-bit
    // indices and division
    for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < (unsigned)(AM_NT * nc); e += gridDim.x * blockDim.x) {
        const int i = (int)(e / (unsigned)nc), q = (int)(e - (unsigned)i * (unsigned)nc);
        const double lt = (0.5 + i) * s.ldt;
        const double ai = s.ls * s.ls + 4. * s.lalpha * lt;
        if (q < nx) {
            const double lx = (p.origin[0] + ((double)q + 0.5) * p.cellSize) - s.xnow;
            const double u = lx + m.lv * lt;
            const Real xv = (Real)exp(-(u * u) / ai);
            X[(long long)i * nx + q] = xv;
            if (sizeof(Real) == 4 && a.d.am_ximg && q >= 1 && q <= g.gx) {
                // the tensor-core operand image (am_tc.cu): 2^14 X as FP16 head
                // and remainder, [x tile][16-node K-step][head, remainder][128 x
                // 16], K-major no-swizzle core matrices (offsets in halves)
                const int r = (q - 1) & 127, xt = (q - 1) >> 7, ks = i >> 4, k = i & 15;
                const long long blk = ((long long)xt * (AM_NT / 16) + ks) * 2 * 2048;
                const int off = (r >> 3) * 128 + (k >> 3) * 64 + (r & 7) * 8 + (k & 7);
                const float xs = (float)xv * 16384.f;
                const __half hi = __float2half_rn(xs);
                __half *img = (__half *)a.d.am_ximg;
                img[blk + off] = hi;
                img[blk + 2048 + off] = __float2half_rn(xs - __half2float(hi));
            }
        } else if (q < nx + ny) {
            const int J = q - nx;
            const double ly = (p.origin[1] + ((double)J + 0.5) * p.cellSize) - s.ynow;
            const Real yv = (Real)exp(-(ly * ly) / ai);
            Y[(long long)i * ny + J] = yv;
            // the tensor-core producers' copy, nodes contiguous per row (am_tc.cu)
            if (sizeof(Real) == 4 && a.d.am_ximg) am_yt(a.d.am_ximg, g.gx)[(long long)J * AM_NT + i] = (float)yv;
        } else {
            const int K = q - nx - ny;
            const double rz = p.origin[2] + ((double)(K + p.kz0) + 0.5) * p.cellSize;
            const double lz = rz - s.znow;
            const double Tlocal = sqrt(s.lalpha * lt) * ai;
            const Real zv = (Real)(s.ldt * exp(-(lz * lz / (4. * s.lalpha * lt))) / Tlocal);
            Z[(long long)i * nz + K] = zv;
            if (sizeof(Real) == 4 && a.d.am_ximg)
                am_zt(a.d.am_ximg, g.gx, g.gy)[(long long)K * AM_NT + i] = (float)zv;
            if (i == 0) zon[K] = (rz <= s.znow + p.cellSize) ? 1 : 0;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *am_tab_step(zon, nz) = ctl->timestep + 1;
        if (sizeof(Real) == 4) *am_tab_sb(zon, nz) = (float)am_b_scale(s);
    }
}

// T over tiles of (XL MX) x-cells by (G MY) (y, z) rows, G = 256 / XL: each
// thread keeps MX x MY sums (x cells XL apart, MY consecutive rows), streaming
// the node axis through shared memory 16 nodes at a time; per node a thread
// reads MX X values (consecutive across the x lanes, no bank conflicts) and
// MY YZ products (the same for the lanes of one row group) for MX MY fused
// multiply-adds.
template <typename Real>
struct AmTile;
template <>
struct AmTile<double> {
    static constexpr int XL = 16, MX = 4, MY = 8, MINB = 2;
};
template <>
struct AmTile<float> {
    static constexpr int XL = 16, MX = 4, MY = 8, MINB = 2;
};
constexpr int AMC_CH = 16, AMC_NT = 256;

template <typename Real>
__global__ void __launch_bounds__(AMC_NT, AmTile<Real>::MINB) k_am_contract(KernelArgs a, AmParams m)
{
    using TL = AmTile<Real>;
    constexpr int XL = TL::XL, MX = TL::MX, MY = TL::MY, G = AMC_NT / XL;
    constexpr int TX = XL * MX, TR = G * MY;
    const Ctl *ctl = a.d.ctl;
    if (stalled(ctl)) return;
    const Geo &g = a.g;
    const Phys &p = a.p;
    const int nx = g.gx + 2, ny = g.gy + 2, nz = g.gz + 2;
    const Real *X = (const Real *)a.d.am_tab, *Y = X + (long long)AM_NT * nx, *Z = Y + (long long)AM_NT * ny;
    const int *zon = (const int *)(Z + (long long)AM_NT * nz);
    __shared__ __align__(16) Real sX[AMC_CH][TX];
    __shared__ __align__(16) Real sYZ[AMC_CH][TR];
    const int tid = threadIdx.x, xl = tid % XL, grp = tid / XL;
    const int x0 = blockIdx.x * TX;
    const long long r0 = (long long)blockIdx.y * TR;  // row = K * ny + J
    const long long nrows = (long long)ny * nz;
    __shared__ int s_any;
    if (tid == 0) s_any = 0;
    __syncthreads();
    for (int q = tid; q < TR; q += AMC_NT)
        if (r0 + q < nrows && zon[(r0 + q) / ny]) s_any = 1;
    __syncthreads();
    Real acc[MX][MY];
#pragma unroll
    for (int u = 0; u < MX; u++)
#pragma unroll
        for (int q = 0; q < MY; q++) acc[u][q] = 0;
    if (s_any) {
        // each thread stages the same x columns and (y, z) rows of every
        // chunk: their table offsets are fixed for the whole sum
        constexpr int XSTEP = AMC_NT / TX;
        const int xx = tid % TX, xi0 = tid / TX;
        const bool xin = x0 + xx < nx;
        const Real *Xp = X + (x0 + xx);
        static_assert(AMC_NT % TR == 0 || TR % AMC_NT == 0, "row staging");
        constexpr int YSTEP = TR >= AMC_NT ? 1 : AMC_NT / TR;     // nodes apart
        constexpr int RPT = TR >= AMC_NT ? TR / AMC_NT : 1;       // rows per thread
        const int yi0 = TR >= AMC_NT ? 0 : tid / TR;
        const Real *Yp[RPT];
        const Real *Zp[RPT];
        bool rin[RPT];
#pragma unroll
        for (int w = 0; w < RPT; w++) {
            const int rl = (tid % (TR < AMC_NT ? TR : AMC_NT)) + w * AMC_NT;
            const long long row = r0 + rl;
            rin[w] = row < nrows;
            const int Kr = rin[w] ? (int)(row / ny) : 0, Jr = rin[w] ? (int)(row - (long long)Kr * ny) : 0;
            Yp[w] = Y + Jr;
            Zp[w] = Z + Kr;
        }
        for (int i0 = 0; i0 < AM_NT; i0 += AMC_CH) {
#pragma unroll
            for (int ii = xi0; ii < AMC_CH; ii += XSTEP)
                sX[ii][xx] = xin ? Xp[(long long)(i0 + ii) * nx] : (Real)0;
#pragma unroll
            for (int ii = yi0; ii < AMC_CH; ii += YSTEP)
#pragma unroll
                for (int w = 0; w < RPT; w++) {
                    const int rl = (tid % (TR < AMC_NT ? TR : AMC_NT)) + w * AMC_NT;
                    sYZ[ii][rl] = rin[w] ? Yp[w][(long long)(i0 + ii) * ny] * Zp[w][(long long)(i0 + ii) * nz]
                                         : (Real)0;
                }
            __syncthreads();
#pragma unroll 4
            for (int ii = 0; ii < AMC_CH; ii++) {
                Real xv[MX], yz[MY];
#pragma unroll
                for (int u = 0; u < MX; u++) xv[u] = sX[ii][xl + XL * u];
#pragma unroll
                for (int q = 0; q < MY; q++) yz[q] = sYZ[ii][grp * MY + q];
#pragma unroll
                for (int u = 0; u < MX; u++)
#pragma unroll
                    for (int q = 0; q < MY; q++) acc[u][q] = fma(xv[u], yz[q], acc[u][q]);
            }
            __syncthreads();
        }
    }
    const AmStep s = am_step(p, m, ctl->timestep + 1);
#pragma unroll
    for (int q = 0; q < MY; q++) {
        const long long row = r0 + grp * MY + q;
        if (row >= nrows) break;
        const int K = (int)(row / ny), J = (int)(row - (long long)K * ny);
        const bool on = zon[K] != 0;
#pragma unroll
        for (int u = 0; u < MX; u++) {
            const int x = x0 + xl + XL * u;
            if (x >= nx) continue;
            const long long c = (long long)K * g.sz + (long long)J * g.sy + x;
            const double T = on ? s.liniT + s.Tfront * (double)acc[u][q] : 0.0;
            a.d.T[c] = T;
            if (a.d.lsindex && T > p.Tliq) a.d.lsindex[c] = 1;
        }
    }
}

// --------------------------------------------------------------- nucleation
// cell_nucleation (grain.c:1222-1285) over the sparse site list: a cell with
// an infinite threshold can never pass the test, so only sites are tested.
// Each block keeps its candidates in site order (cand_stage) with a count,
// so that k_act can gather them in (emulated rank, local raster) order.
constexpr int NUC_NT = 256;
template <typename Real>
__device__ __forceinline__ void nuc_body(const KernelArgs &a, int bid)
{
    Ctl *ctl = a.d.ctl;
    if (stalled(ctl)) return;
    __shared__ int sh[NUC_NT / 32];
    const Geo &g = a.g;
    const Phys &p = a.p;
    long long s = bid * (long long)NUC_NT + threadIdx.x;
    int hit = 0;
    if (s < a.d.nsites) {
        unsigned long long ts = ctl->timestep + 1;
        long long c = a.d.site_cell[s];
        // the site's grain id, liquid concentration, threshold and (AM)
        // temperature are loaded together, before the grain-id test
        const Real *cl = (const Real *)a.d.cl[(int)(ctl->timestep & 1ULL)];
        const int grc = a.d.gr[c];
        const double clc = (double)cl[c];
        const double thr = (double)a.d.site_thr[s];
        const double Tarr = p.temp_mode == 2 ? (a.d.T32 ? (double)a.d.T32[c] : a.d.T[c]) : 0.0;
        if (grc <= 0) {
            double Ttemp = Tarr;
            if (p.temp_mode != 2) {
                const long long K = c / g.sz, J = (c % g.sz) / g.sy;
                Ttemp = temp_cell(p, a.d.T, a.d.T32, c, J, K, ts);
            }
            int layerno = 1, initnuc = 1;
            if (p.am) {
                double sim_time = (double)ts * p.ts_delt;
                if (p.amlayer == 1) layerno = 1;
                else if (p.amlayer > 1 && a.d.lsindex[c] == 1) layerno = 1;
                else layerno = 0;
                if (sim_time <= 1e-4) initnuc = 1;
                else if (Ttemp >= p.Tsol) initnuc = 1;
                else initnuc = 0;
            }
            if (layerno && initnuc) {
                double Tunder = p.Tliq - Ttemp;
                double m = p.ma * Ttemp * Ttemp + p.mb * Ttemp + p.mc;
                // the FP32 form stores cl - Cinit
                Tunder += m * ((sizeof(Real) == 8) ? (clc - p.cinit) : clc);
                if (Tunder > thr) hit = 1;
            }
        }
    }
    int tot;
    int pos = block_exclusive_scan<NUC_NT>(hit, tot, sh);
    if (hit) a.d.cand_stage[bid * (long long)NUC_NT + pos] = (int)s;
    if (threadIdx.x == 0) {
        a.d.nuc_blk_cnt[bid] = tot;
        if (tot) atomicAdd(&ctl->ncand, tot);
    }
}

template <typename Real>
__global__ void __launch_bounds__(NUC_NT) k_nuc(KernelArgs a)
{
    nuc_body<Real>(a, blockIdx.x);
}

__device__ long long find_key(const long long *keys, long long n, long long key)
{
    long long lo = 0, hi = n - 1;
    while (lo <= hi) {
        long long mid = (lo + hi) >> 1;
        long long k = keys[mid];
        if (k == key) {
            while (mid > 0 && keys[mid - 1] == key) mid--;
            return mid;
        }
        if (k < key) lo = mid + 1;
        else hi = mid - 1;
    }
    return -1;
}

// activateNewGrains + createGrains (grain.c:840-916, 347-425).  Candidates
// are gathered in site order, which is (emulated rank, local raster) order,
// so candidate i gets grain id num_grains + i, as the rank-ordered
// Allgatherv displacements give (grain.c:892-904); the k-th candidate of
// rank r without a deck-defined orientation takes that rank's k-th
// pre-drawn orientation.  More candidates than MaxTotGrains leaves room
// for is the reference's createGrains error (grain.c:363-366): nindex2
// replaces the capped count (grain.c:1318), so the cap never holds.
// One CTA; every phase is parallel over candidates or ranks.
constexpr int ACT_NT = 1024;

// Ordered gather of the per-block candidate lists into cand[0, C), then per
// candidate its orientation source and the prefix count of random draws
// (cand_ex), per rank its first candidate and its number of draws.
template <int NT>
__device__ __forceinline__ void act_gather(const KernelArgs &a, int C, int *need, int *first, int *sh)
{
    const Phys &p = a.p;
    const int nr = a.g.nranks;
    int *ex = a.d.cand_ex;
    for (int r = threadIdx.x; r < nr; r += NT) need[r] = 0, first[r] = -1;
    int off = 0;
    for (int base = 0; base < a.d.nuc_blocks; base += NT) {
        int b = base + threadIdx.x;
        int n = (b < a.d.nuc_blocks) ? a.d.nuc_blk_cnt[b] : 0;
        int tot;
        int pos = off + block_exclusive_scan<NT>(n, tot, sh);
        for (int i = 0; i < n; i++) a.d.cand[pos + i] = a.d.cand_stage[(long long)b * NUC_NT + i];
        off += tot;
    }
    __syncthreads();
    int run = 0;
    for (int base = 0; base < C; base += NT) {
        int i = base + threadIdx.x;
        int rnd = 0, r = 0;
        if (i < C) {
            long long cell = a.d.site_cell[a.d.cand[i]];
            r = a.d.site_rank[a.d.cand[i]];
            rnd = (p.use_orientation && find_key(a.d.nucpt_key, a.d.n_nucpt, cell) < 0) ? 1 : 0;
            if (i == 0 || a.d.site_rank[a.d.cand[i - 1]] != r) first[r] = i;
            if (rnd) atomicAdd(&need[r], 1);
        }
        int tot;
        int e = run + block_exclusive_scan<NT>(rnd, tot, sh);
        if (i < C) ex[i] = e;
        run += tot;
    }
    __syncthreads();
}

// Some rank lacks pre-drawn orientations for its draws of this step (block-wide).
template <int NT>
__device__ __forceinline__ bool act_short(const KernelArgs &a, const int *need)
{
    int short_rng = 0;
    for (int r = threadIdx.x; r < a.g.nranks; r += NT)
        if (a.d.rng_used[r] + need[r] > a.d.rng_cap) short_rng = 1;
    return __syncthreads_or(short_rng) != 0;
}

// Grain id0 + i for candidate i: gr, rotation and record; with rows, the
// record as the other slabs of a split domain receive it.
template <int NT>
__device__ __forceinline__ void act_assign(const KernelArgs &a, int C, long long id0, unsigned long long ts,
                                           const int *first, SlabRow *rows)
{
    const Phys &p = a.p;
    const Geo &g = a.g;
    const int *ex = a.d.cand_ex;
    for (int i = threadIdx.x; i < C; i += NT) {
        const int s = a.d.cand[i];
        if (!in_bounds(a.d.ctl, s, a.d.nsites)) continue;
        const long long cell = a.d.site_cell[s];
        const int r = a.d.site_rank[s];
        const long long id = id0 + i;
        if (!in_bounds(a.d.ctl, cell, g.N) || !in_bounds(a.d.ctl, r, g.nranks) ||
            !in_bounds(a.d.ctl, id, (long long)p.max_grains + 1))
            continue;
        a.d.gr[cell] = (int)id;
        GrainLog lg;
        lg.cell = cell;
        lg.timestep = ts;
        lg.rank = r + a.d.rank0;
        lg.thr = a.d.site_thr[s];
        lg.pad = 0;
        const double *rot;
        long long j = find_key(a.d.nucpt_key, a.d.n_nucpt, cell);
        if (j >= 0) {
            rot = a.d.nucpt_rot + 9 * j;
            lg.kind = 0;
            lg.aux = a.d.nucpt_entry[j];
        } else if (p.use_orientation) {
            // this rank's draws before candidate i
            const int k = a.d.rng_used[r] + (ex[i] - ex[first[r]]);
            if (!in_bounds(a.d.ctl, k, a.d.rng_cap)) continue;
            rot = a.d.rng_rot + ((long long)r * a.d.rng_cap + k) * 9;
            lg.kind = 1;
            lg.aux = a.d.rng_base[r] + k;
        } else {
            rot = a.d.zero_rot;
            lg.kind = 2;
            lg.aux = 0;
        }
        if (a.d.n_inj > 0) {
            long long q = find_key(a.d.inj_key, a.d.n_inj, cell);
            if (q >= 0) rot = a.d.inj_rot + 9 * q;
        }
        double *dst = a.d.grain_rot + 9 * id;
        for (int e = 0; e < 9; e++) dst[e] = rot[e];
        a.d.grain_log[id] = lg;
        if (rows) {
            SlabRow &row = rows[i];
            for (int e = 0; e < 9; e++) row.rot[e] = rot[e];
            const long long K = cell / g.sz, J = (cell % g.sz) / g.sy, I = cell % g.sy;
            lg.cell = (K + p.kz0) * g.rsz + J * g.rsy + I;
            row.lg = lg;
        }
    }
}

template <int NT>
__device__ __forceinline__ void act_body(const KernelArgs &a, int *rank_scratch)
{
    Ctl *ctl = a.d.ctl;
    if (stalled(ctl)) return;
    __shared__ int sh[NT / 32];
    __shared__ int s_abort;
    const int C = ctl->ncand;
    const unsigned long long ts = ctl->timestep + 1;
    if (threadIdx.x == 0) ctl->list_ticket = 0;  // k_list block order of this step
    if (C == 0) {
        if (threadIdx.x == 0) {
            ctl->timestep = ts;
            ctl->new_grains = 0;
        }
        return;
    }
    const Phys &p = a.p;
    const int nr = a.g.nranks;
    int *need = rank_scratch;        // random draws per rank
    int *first = rank_scratch + nr;  // first candidate of each rank
    if (threadIdx.x == 0) s_abort = 0;
    act_gather<NT>(a, C, need, first, sh);
    if (threadIdx.x == 0) {
        if ((unsigned long long)(ctl->num_grains + (long long)C) > p.max_grains + 1) {
            ctl->status = MMS_ERR_GRAIN_OVERFLOW;
            atomicExch(&ctl->stall, (int)STALL_ERROR);
            s_abort = 1;
        }
    }
    __syncthreads();
    if (s_abort) return;
    if (act_short<NT>(a, need)) {
        // refill on the host, then this kernel runs again with the same
        // candidates (nothing has been written yet)
        if (threadIdx.x == 0) {
            ctl->stall_step = ts;
            atomicExch(&ctl->stall, (int)STALL_RNG);
        }
        return;
    }
    const long long num_grains = ctl->num_grains;
    act_assign<NT>(a, C, num_grains, ts, first, nullptr);
    __syncthreads();
    for (int r = threadIdx.x; r < nr; r += NT)
        if (need[r]) atomicMax(&ctl->rng_used_max, a.d.rng_used[r] += need[r]);
    if (threadIdx.x == 0) {
        ctl->num_grains = (int)(num_grains + C);
        ctl->new_grains = C;
        ctl->ncand = 0;
        ctl->timestep = ts;
    }
}

// Slab of a split domain, before the first exchange: this slab's half of
// activation (gather, draws needed), published as {candidates, short of
// draws} for every slab to see.
__global__ void __launch_bounds__(ACT_NT) k_act_local(KernelArgs a)
{
    Ctl *ctl = a.d.ctl;
    if (stalled(ctl)) return;
    __shared__ int sh[ACT_NT / 32];
    const int C = ctl->ncand;
    if (threadIdx.x == 0) ctl->list_ticket = 0;
    if (C > a.d.slab_cap) {  // more candidates than the row buffer holds
        if (threadIdx.x == 0) raise_error(ctl, MMS_ERR_SLAB_CAPACITY);
        return;
    }
    int short_rng = 0;
    if (C > 0) {
        int *need = a.d.act_scratch, *first = a.d.act_scratch + a.g.nranks;
        act_gather<ACT_NT>(a, C, need, first, sh);
        short_rng = act_short<ACT_NT>(a, need) ? 1 : 0;
    }
    if (threadIdx.x == 0) {
        a.d.x1_send[0] = C;
        a.d.x1_send[1] = short_rng;
    }
}

// Slab of a split domain, after the first exchange: grain ids continue
// over the slabs in slab order, which is emulated-rank order because every
// slab holds whole layers of subblocks.  Every slab takes the same
// decision on overflow and on a shortage of draws anywhere, so a stalled
// step stalls every slab at the same kernel.
__global__ void __launch_bounds__(ACT_NT) k_act_slab(KernelArgs a)
{
    Ctl *ctl = a.d.ctl;
    if (stalled(ctl)) return;
    __shared__ int s_abort;
    const unsigned long long ts = ctl->timestep + 1;
    const int S = a.d.nslabs;
    long long total = 0, off = 0;
    int any_short = 0;
    for (int s = 0; s < S; s++) {
        const int c = a.d.x1_recv[2 * s];
        if (s < a.d.slab) off += c;
        total += c;
        any_short |= a.d.x1_recv[2 * s + 1];
    }
    const int C = ctl->ncand;
    if (threadIdx.x == 0) {
        s_abort = 0;
        if (total > 0 && (unsigned long long)(ctl->num_grains + total) > a.p.max_grains + 1) {
            ctl->status = MMS_ERR_GRAIN_OVERFLOW;
            atomicExch(&ctl->stall, (int)STALL_ERROR);
            s_abort = 1;
        } else if (any_short) {
            ctl->stall_step = ts;
            atomicExch(&ctl->stall, (int)STALL_RNG);
            s_abort = 1;
        }
    }
    __syncthreads();
    if (s_abort) return;
    const long long num_grains = ctl->num_grains;
    if (C > 0) {
        const int nr = a.g.nranks;
        const int *need = a.d.act_scratch, *first = a.d.act_scratch + nr;
        act_assign<ACT_NT>(a, C, num_grains + off, ts, first, a.d.x2_send);
        __syncthreads();
        for (int r = threadIdx.x; r < nr; r += ACT_NT)
            if (need[r]) atomicMax(&ctl->rng_used_max, a.d.rng_used[r] += need[r]);
    }
    if (threadIdx.x == 0) {
        ctl->num_grains = (int)(num_grains + total);
        ctl->new_grains = (int)total;
        ctl->ncand = 0;
        ctl->timestep = ts;
    }
}

// Slab of a split domain, after the second exchange: rotations and records
// of the grains the other slabs created this step.
__global__ void __launch_bounds__(256) k_slab_merge(KernelArgs a)
{
    const Ctl *ctl = a.d.ctl;
    if (stalled(ctl)) return;
    const int S = a.d.nslabs;
    long long total = 0;
    for (int s = 0; s < S; s++) total += a.d.x1_recv[2 * s];
    const long long base = ctl->num_grains - total;
    long long off = 0;
    for (int s = 0; s < S; s++) {
        const int c = a.d.x1_recv[2 * s];
        if (s != a.d.slab) {
            const int n = c < a.d.slab_cap ? c : a.d.slab_cap;
            const SlabRow *rows = a.d.x2_recv + (long long)s * a.d.slab_cap;
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                const long long id = base + off + i;
                double *dst = a.d.grain_rot + 9 * id;
                for (int e = 0; e < 9; e++) dst[e] = rows[i].rot[e];
                GrainLog lg = rows[i].lg;
                lg.kind |= GL_REMOTE;
                a.d.grain_log[id] = lg;
            }
        }
        off += c;
    }
}

__global__ void __launch_bounds__(ACT_NT) k_act(KernelArgs a, int *rank_scratch)
{
    act_body<ACT_NT>(a, rank_scratch);
}

// Nucleation and activation in one launch: every block tests its sites as
// k_nuc does; the block that finishes last (a counter in the control block,
// after a fence in every thread that wrote candidates) then runs
// activateNewGrains over the candidates of all blocks, as k_act would.
template <typename Real>
__global__ void __launch_bounds__(NUC_NT) k_nuc_act(KernelArgs a)
{
    Ctl *ctl = a.d.ctl;
    if (stalled(ctl)) return;  // nothing in this launch changes the stall state before the last block
    nuc_body<Real>(a, blockIdx.x);
    __shared__ int s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(&ctl->nuc_done, 1) == (int)gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x == 0) ctl->nuc_done = 0;
    act_body<NUC_NT>(a, a.d.act_scratch);
}

// ---------------------------------------------------------------- curvature
// x^1.5 for x >= 1, to the nearest double: the product x * sqrt(x) carried
// exactly as a pair (fma gives the rounding error of the product and the
// residual x - s^2 of the rounded square root s), so the one final rounding
// matches a correctly rounded pow(x, 1.5) except when the exact value lies
// within about 1e-16 ulp of a rounding boundary.
__device__ __forceinline__ double pow_1_5(double x)
{
    const double s = sqrt(x);
    const double res = fma(-s, s, x);     // x - s^2, exact
    const double e = res / (2.0 * s);     // sqrt(x) - s to first order
    const double ph = x * s;
    const double pl = fma(x, s, -ph);     // x s - ph, exact
    return ph + (pl + x * e);
}

// sb_curvature (curvature.c:31-405) on each emulated rank's local range
// k,j,i in [2, dim-1], reading fs as it stands before fs_change.
template <typename Real>
__global__ void k_curv(KernelArgs a)
{
    const Ctl *ctl = a.d.ctl;
    if (stalled(ctl)) return;
    const Geo &g = a.g;
    long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long total = (long long)g.nranks * g.sbcells;
    if (v >= total) return;
    int r = (int)(v / g.sbcells);
    long long l = v % g.sbcells;
    int i = (int)(l % g.sbx) + 1, j = (int)((l / g.sbx) % g.sby) + 1, k = (int)(l / ((long long)g.sbx * g.sby)) + 1;
    int rx = r % g.nsbx, ry = (r / g.nsbx) % g.nsby, rz = r / (g.nsbx * g.nsby);
    long long idx = (long long)(rz * g.sbz + k) * g.sz + (long long)(ry * g.sby + j) * g.sy + (rx * g.sbx + i);
    const int dimx = g.sbx, dimy = g.sby, dimz = g.sbz;
    if (i < 2 || i > dimx - 1 || j < 2 || j > dimy - 1 || k < 2 || k > dimz - 1) return;
    const Real *fsr = (const Real *)a.d.fs[(int)((ctl->timestep - 1) & 1ULL)];
    const int *gr = a.d.gr;
    double *curv = a.d.curv;
    auto fs = [&](long long q) { return (double)fsr[q]; };
    curv[idx] = 0.0;
    if (gr[idx] <= 0 || fs(idx) == 0) return;
    const long long jgap = g.sy, kgap = g.sz;
    int nbindex = gr[idx + 1] + gr[idx + jgap] + gr[idx - 1] + gr[idx - jgap] + gr[idx + kgap] + gr[idx - kgap];
    if (!nbindex) return;
    const int alpha = 2, beta = 4;
    long long idl = idx + 1, idr = idx - 1, idf = idx + jgap, idb = idx - jgap;
    long long idu = idx + kgap, idd = idx - kgap;
    long long idur = idr + kgap, idul = idl + kgap, iddr = idr - kgap, iddl = idl - kgap;
    long long idfr = idf - 1, idfl = idf + 1, idbr = idb - 1, idbl = idb + 1;
    long long idub = idb + kgap, iduf = idf + kgap, iddf = idf - kgap, iddb = idb - kgap;
    long long idufr = iduf - 1, idufl = iduf + 1, idubr = idub - 1, idubl = idub + 1;
    long long iddbr = iddb - 1, iddbl = iddb + 1, iddfr = iddf - 1, iddfl = iddf + 1;
    double fsl = (fs(idufl) + fs(idubl) + fs(iddbl) + fs(iddfl) +
                  alpha * (fs(idul) + fs(iddl) + fs(idfl) + fs(idbl)) + beta * fs(idl)) / (1 + 4 * alpha + beta);
    double fsr_ = (fs(idufr) + fs(idubr) + fs(iddbr) + fs(iddfr) +
                   alpha * (fs(idur) + fs(iddr) + fs(idfr) + fs(idbr)) + beta * fs(idr)) / (1 + 4 * alpha + beta);
    double fsf = (fs(idufl) + fs(idufr) + fs(iddfr) + fs(iddfl) +
                  alpha * (fs(idfl) + fs(idfr) + fs(iduf) + fs(iddf)) + beta * fs(idf)) / (1 + 4 * alpha + beta);
    double fsb = (fs(idubr) + fs(idubl) + fs(iddbl) + fs(iddbr) +
                  alpha * (fs(idbl) + fs(idbr) + fs(idub) + fs(iddb)) + beta * fs(idb)) / (1 + 4 * alpha + beta);
    // the reference weights fs[idl] here (curvature.c:176); corrected: fs[idu]
    const bool fixed = a.p.curv_fixed != 0;
    double fsu = (fs(idufl) + fs(idufr) + fs(idubr) + fs(idubl) +
                  alpha * (fs(idul) + fs(idur) + fs(idub) + fs(iduf)) + beta * fs(fixed ? idu : idl)) /
                 (1 + 4 * alpha + beta);
    double fsd = (fs(iddbr) + fs(iddbl) + fs(iddfl) + fs(iddfr) +
                  alpha * (fs(iddr) + fs(iddl) + fs(iddf) + fs(iddb)) + beta * fs(idd)) / (1 + 4 * alpha + beta);
    double nx = (fsl - fsr_) / 2.0, ny = (fsf - fsb) / 2.0, nz = (fsu - fsd) / 2.0;
    double nall = sqrt(nx * nx + ny * ny + nz * nz);
    // the reference normalises only a zero normal (curvature.c:194) and picks
    // a height direction only when a component is exactly zero
    // (curvature.c:203); corrected: a non-zero normal, and always
    if (fixed ? (nall != 0.0) : !(nall)) {
        nx = nx / nall;
        ny = ny / nall;
        nz = nz / nall;
    }
    int nor_dir = 0;
    if (fixed || !(nx) || !(ny) || !(nz)) {
        if ((fabs(nx) >= fabs(ny)) && (fabs(nx) >= fabs(nz))) nor_dir = 1;
        else if ((fabs(ny) >= fabs(nz)) && (fabs(ny) >= fabs(nx))) nor_dir = 2;
        else if ((fabs(nz) >= fabs(ny)) && (fabs(nz) >= fabs(nx))) nor_dir = 3;
    }
    long long st, a1, a2, b1, b2, c11, c12, c21, c22;
    double ncomp;
    int pos, dim;
    if (nor_dir == 3) {
        ncomp = nz; pos = k; dim = dimz; st = kgap;
        a1 = idf; a2 = idb; b1 = idl; b2 = idr; c11 = idfl; c12 = idfr; c21 = idbl; c22 = idbr;
    } else if (nor_dir == 2) {
        ncomp = ny; pos = j; dim = dimy; st = jgap;
        a1 = idu; a2 = idd; b1 = idl; b2 = idr; c11 = idul; c12 = idur; c21 = iddl; c22 = iddr;
    } else if (nor_dir == 1) {
        ncomp = nx; pos = i; dim = dimx; st = 1;
        a1 = idu; a2 = idd; b1 = idf; b2 = idb; c11 = iduf; c12 = idub; c21 = iddf; c22 = iddb;
    } else {
        return;
    }
    double gamma = (acos(fabs(ncomp)) < 0.8) ? 0.0 : 0.2;
    int t = (((pos + 2) <= dim) && (pos - 2) >= 1) ? 3 : 1;
    double h = 0, hA1 = 0, hA2 = 0, hB1 = 0, hB2 = 0, hC11 = 0, hC12 = 0, hC22 = 0, hC21 = 0;
    for (int n = -t; n <= t; n++) {
        h += fs(idx + st * n);
        hA1 += fs(a1 + st * n);
        hA2 += fs(a2 + st * n);
        hB1 += fs(b1 + st * n);
        hB2 += fs(b2 + st * n);
        hC11 += fs(c11 + st * n);
        hC12 += fs(c12 + st * n);
        hC22 += fs(c22 + st * n);
        hC21 += fs(c21 + st * n);
    }
    double cs = a.p.cellSize;
    double hx = (gamma * (hC11 - hC12) + hB1 - hB2 + gamma * (hC21 - hC22)) / (1 + 2 * gamma) / 2.0;
    double hy = (gamma * (hC11 - hC21) + hA1 - hA2 + gamma * (hC12 - hC22)) / (1 + 2 * gamma) / 2.0;
    double hxx = (gamma * (hC11 - 2 * hA1 + hC12) + hB1 - 2 * h + hB2 + gamma * (hC21 - 2 * hA2 + hC22)) / (cs) / (1 + 2 * gamma);
    double hyy = (gamma * (hC11 - 2 * hB1 + hC21) + hA1 - 2 * h + hA2 + gamma * (hC12 - 2 * hB2 + hC22)) / (cs) / (1 + 2 * gamma);
    double hxy = (hC11 - hC21 - hC12 + hC22) / cs / 4.0;
    curv[idx] = (hxx + hyy + hxx * hy * hy + hyy * hx * hx - 2 * hxy * hx * hy) / pow_1_5((1 + hx * hx + hy * hy));
}

// ------------------------------------------------ diffusion + fs change
// Per cell: sb_diffuse_alloy_decentered (growth.c:69-162) followed by
// fs_change_diffuse (growth.c:220-273) on the same cell, with oce = the ce
// value before diffusion, held in a register (calculate.c:269-280).  The
// neighbour values are read before any cell of this step writes them: cl
// and fs come from the previous step's buffer.

// nb_* in the order +x, -x, +y, -y, +z, -z (growth.c:85-113); one_m[n] is
// (1 - mold) of that neighbour.
//
// FP32 form: ce and cl are stored as deviations from Cinit (conc, nb_cl,
// oce, and the results likewise), so that the liquid, where they stay close
// to Cinit, keeps ~1e-10 wt% absolute resolution instead of float's 5e-7;
// the undercooling T - Tliq is formed in FP64 before rounding, and the
// solute increment dce is the diffusion sum itself rather than the
// difference of two rounded ce values.
// interior: no face of this cell touches the domain halo, so every (1 -
// mold) factor is 1.0 and the multiplication by it (exact) is skipped.
template <typename Real>
__device__ __forceinline__ Real diff_sum(const PhysR<Real> &q, Real conc, Real lspfs, const Real (&nb_cl)[6],
                                         const Real (&nb_fs)[6], const Real (&one_m)[6], bool interior)
{
    Real nbsum = 0;
    if (sizeof(Real) == 4) {
        // FP32 form: the face coefficient rs fs_av + rl (1 - fs_av) written
        // as A + B fs_n with fused multiply-adds
        const float B = 0.5f * ((float)q.rs - (float)q.rl);
        const float A = fmaf(B, (float)lspfs, (float)q.rl);
        float acc = 0.f;
#pragma unroll
        for (int n = 0; n < 6; n++) {
            float r = fmaf(B, (float)nb_fs[n], A);
            if (!interior) r *= (float)one_m[n];
            acc = fmaf(r, (float)nb_cl[n] - (float)conc, acc);
        }
        nbsum = (Real)acc;
    } else if (interior) {
#pragma unroll
        for (int n = 0; n < 6; n++) {
            Real fs_av = (Real)0.5 * (lspfs + nb_fs[n]);
            Real r = (q.rs * fs_av + q.rl * (1 - fs_av));
            nbsum += r * (nb_cl[n] - conc);
        }
    } else {
#pragma unroll
        for (int n = 0; n < 6; n++) {
            Real fs_av = (Real)0.5 * (lspfs + nb_fs[n]);
            Real r = (q.rs * fs_av + q.rl * (1 - fs_av)) * one_m[n];
            nbsum += r * (nb_cl[n] - conc);
        }
    }
    return nbsum;
}

// fs_change_diffuse (growth.c:220-272) of one cell given its diffusion sum.
// The fs change of the FP32 form from dT = T - Tliq and the range test
// (off: T < 1 or T > Tliq), shared by the FP64- and FP32-temperature entries
__device__ __forceinline__ void fs_update_f32(const PhysR<float> &q, const Phys &p, float conc, float lspfs,
                                              float nbsum, float oce, int grc, float dT, bool off, const double *curv,
                                              long long c, float &cen, float &cl_new, float &fs_new, int &gr_new,
                                              int &br)
{
    using Real = float;
    cen = oce + nbsum;
    gr_new = grc;
    Real c_int = q.m_inv * dT;               // c_int - Cinit
    Real Tunder = -dT + q.liq_slope * conc;  // conc = cl - Cinit
    if (grc <= 0 || off) {
        cl_new = cen;
        fs_new = 0;
        gr_new = 0;
        br = BR_RESET;
    } else if (lspfs == (Real)1.0 && (Tunder >= (Real)0.0)) {
        cl_new = cen * q.k_inv + q.c0k;      // ce / k - Cinit
        fs_new = lspfs;
        br = BR_KEEP;
    } else {
        if (p.tip_curv) c_int = q.m_inv * (dT + q.gibbs * (Real)curv[c]);
        // dce = the diffusion sum; dcl (u - 1/u terms) and dfs with the
        // dce terms of growth.c:257-261 cancelled algebraically:
        // dcl u - dce = (c_int - cl) 2 D_xt u
        const float dce = (float)nbsum;
        const float u = 1.f - (float)q.km * (float)lspfs;
        const float t2 = ((float)c_int - (float)conc) * (2.f * (float)q.D_xt);
        const float dcl = t2 + __fdividef(dce, u);
        const float dfs = __fdividef(t2 * u * (float)q.km_inv, (float)conc + (float)q.cinit);
        cl_new = conc + dcl;
        fs_new = lspfs + dfs;
        br = ((Real)1.0 < fs_new) ? BR_CLAMP : BR_GROW;
        fs_new = ((Real)1.0 < fs_new) ? (Real)1.0 : fs_new;
        if (fs_new < (Real)0.) {
            fs_new = 0.;
            gr_new = 0;
            cl_new = cen;
            br = BR_NEG;
        }
    }
}

// FP32 form with a temperature held in FP32 (the AM model's array): the
// range test on that value exactly as fs_update makes it (x > Tliq exactly
// when x > Tliq rounded down to FP32) and T - Tliq through Tliq's FP32 head
// and remainder, with no FP32-FP64 conversions
__device__ __forceinline__ void am_dt(const PhysR<float> &q, float Tf, float &dT, bool &off)
{
    dT = __fsub_rn(__fsub_rn(Tf, q.tliq_h), q.tliq_l);
    off = Tf < 1.f || Tf > q.tliq_rd;
}

template <typename Real>
__device__ __forceinline__ void fs_update(const PhysR<Real> &q, const Phys &p, Real conc, Real lspfs, Real nbsum,
                                          Real oce, int grc, double Td, const double *curv, long long c, Real &cen,
                                          Real &cl_new, Real &fs_new, int &gr_new, int &br, bool t32 = false)
{
    cen = oce + nbsum;
    gr_new = grc;
    if constexpr (sizeof(Real) == 8) {
        // fs_change_diffuse, growth.c:220-272, operation for operation
        const Real Tcell = (Real)Td;
        Real c_int = q.cinit + q.m_inv * (Tcell - q.Tliq);
        Real Tunder = q.Tliq - Tcell;
        Tunder += q.liq_slope * (conc - q.cinit);
        if (grc <= 0 || Td < 1.0 || Td > p.Tliq) {
            cl_new = cen;
            fs_new = 0;
            gr_new = 0;
            br = BR_RESET;
        } else if (lspfs == (Real)1.0 && (Tunder >= (Real)0.0)) {
            cl_new = cen * q.k_inv;
            fs_new = lspfs;
            br = BR_KEEP;
        } else {
            if (p.tip_curv) c_int = q.cinit + q.m_inv * (Tcell - q.Tliq + q.gibbs * (Real)curv[c]);
            Real dce = cen - oce;
            Real dcl = (c_int - conc) * q.D_xt * 2 + dce / (1 - q.km * lspfs);
            Real dfs = (dcl * ((Real)1. - q.km * lspfs) - dce) * q.km_inv / conc;
            cl_new = conc + dcl;
            fs_new = lspfs + dfs;
            br = ((Real)1.0 < fs_new) ? BR_CLAMP : BR_GROW;
            fs_new = ((Real)1.0 < fs_new) ? (Real)1.0 : fs_new;
            if (fs_new < (Real)0.) {
                fs_new = 0.;
                gr_new = 0;
                cl_new = cen;
                br = BR_NEG;
            }
        }
    } else {
        // t32: Td holds the value of an FP32 temperature array (the AM
        // model), whose every path takes the FP32-temperature form of the
        // test and the difference
        float dT;
        bool off;
        if (t32) {
            am_dt(q, (float)Td, dT, off);
        } else {
            dT = (float)(Td - p.Tliq);
            off = Td < 1.0 || Td > p.Tliq;
        }
        fs_update_f32(q, p, conc, lspfs, nbsum, oce, grc, dT, off, curv, c, cen, cl_new, fs_new, gr_new, br);
    }
}

template <typename Real>
__device__ __forceinline__ void cell_update(const PhysR<Real> &q, const Phys &p, Real conc, Real lspfs,
                                            const Real (&nb_cl)[6], const Real (&nb_fs)[6],
                                            const Real (&one_m)[6], bool interior, Real oce, int grc,
                                            double Td, const double *curv, long long c, Real &cen,
                                            Real &cl_new, Real &fs_new, int &gr_new, int &br, bool t32 = false)
{
    fs_update<Real>(q, p, conc, lspfs, diff_sum<Real>(q, conc, lspfs, nb_cl, nb_fs, one_m, interior), oce, grc, Td,
                    curv, c, cen, cl_new, fs_new, gr_new, br, t32);
}

constexpr int DTX = 32, DTY = 8;

// TMA-fed variant.  A CTA of 32 x 8 threads owns a (32 CPT) x 8 column of
// cells and marches up a z-chunk: one cell per thread (CPT = 1,
// stencil_tile) or two adjacent cells per thread (CPT = 2,
// stencil_tile_pair), which read their cells and neighbours as 8- or
// 16-byte words of shared memory and write them as such words of global
// memory.  Planes of cl and fs with their x/y halo (and ce, gr without) are
// brought into a TS-deep shared-memory ring by cp.async.bulk.tensor, one
// mbarrier per slot, issued TS-1 planes ahead of the plane being updated.
//
// Alignment.  The fields start 16 - sizeof(element) bytes past a 16-byte
// boundary (field_lead in mms_api.cu) and rows are a multiple of 8
// elements, so interior cell 1 of every row, and every 32nd cell after it,
// is 16-byte aligned.  The tensor maps begin at that boundary, lead =
// 16 / sizeof(element) - 1 elements before the field, with x extent
// gx + 2 + lead: a cl/fs box starts at map x = i0 - 1 (a multiple of the tile
// width) and so holds the tile's first cell i0 at column HX = lead + 1; the
// ce and gr boxes start at i0 itself.
template <typename Real, int CPT>
struct Depth {
    // planes in the ring: deeper for FP32 with one cell per thread, whose
    // planes are smaller; with two cells per thread, five (FP32) or four
    // (FP64) planes, so that four (three) CTAs' rings fit in shared memory
    static constexpr int TS = (sizeof(Real) == 4 && CPT == 1) ? 8 : (CPT == 1 ? 6 : (sizeof(Real) == 4 ? 5 : 4));
    // CTAs per SM the register budget is set for
    static constexpr int MINB = CPT == 1 ? 4 : (sizeof(Real) == 4 ? 4 : 3);
};
constexpr int round128(int b) { return (b + 127) / 128 * 128; }

template <typename Real, int CPT>
struct Stage {
    static constexpr int TX = DTX * CPT;
    // box widths: a multiple of 16 bytes
    static constexpr int EPA = 16 / (int)sizeof(Real);
    static constexpr int LEAD = EPA - 1;                             // field lead (elements)
    static constexpr int HX = EPA;                                   // column of cell i0 in a cl/fs box
    static constexpr int BXH = (TX + HX + 1 + EPA - 1) / EPA * EPA;  // cl, fs: DTY+2 rows, to the right halo
    static constexpr int BXC = TX;                                   // ce: DTY rows from i0
    static constexpr int BXG = TX;                                   // gr (int, lead 3): DTY rows from i0
    static constexpr int CL = round128(BXH * (DTY + 2) * (int)sizeof(Real));
    static constexpr int CE = round128(BXC * DTY * (int)sizeof(Real));
    static constexpr int GR = round128(BXG * DTY * 4);
    static constexpr int BYTES = 2 * CL + CE + GR;
    static constexpr unsigned TX_HALO = 2u * BXH * (DTY + 2) * sizeof(Real);
    static constexpr unsigned TX_CENTER = BXC * DTY * sizeof(Real) + BXG * DTY * 4u;
};

struct TmaMaps {
    CUtensorMap cl[2], fs[2], ce, gr;
};

// Shared-memory state of a stencil CTA, kept across the tiles a persistent
// CTA processes: the ring, one mbarrier per slot (initialised once), the
// per-plane temperatures and the abort flag.
template <int TS>
struct StencilShared {
    unsigned long long bars[TS];
    double sT[64];
    double fsum[DTY];
    int abort;
};

// One (32 CPT) x 8 x zchunk tile (bx, by, bz) of the diffusion + fs-change
// update.  ring: planes this CTA has streamed through its ring before this
// tile, so slot and phase continue across tiles.  part (may be null): the
// tile's sum of the new fraction solid goes to part[2 part_idx] (and 0 to
// part[2 part_idx + 1], the compensation slot of k_reduce_fold).  Returns
// false when a copy did not land within the bound (the error is raised,
// copies in flight are drained).
template <typename Real, int CPT>
__device__ __forceinline__ bool stencil_tile(const KernelArgs &a, const TmaMaps &maps, int zchunk, int bx, int by,
                                             int bz, unsigned char *smem, StencilShared<Depth<Real, CPT>::TS> &sh,
                                             unsigned &ring, double *part = nullptr, long long part_idx = 0)
{
    using L = Stage<Real, CPT>;
    constexpr int TS = Depth<Real, CPT>::TS;
    Ctl *ctl = a.d.ctl;
    unsigned long long *bars = sh.bars;
    const Geo &g = a.g;
    const Phys &p = a.p;
    const unsigned long long ts = ctl->timestep;
    const int pin = (int)((ts - 1) & 1ULL), pout = (int)(ts & 1ULL);
    Real *__restrict__ clO = (Real *)a.d.cl[pout];
    Real *__restrict__ fsO = (Real *)a.d.fs[pout];
    Real *__restrict__ ce = (Real *)a.d.ce;
    int *__restrict__ gr = a.d.gr;
    const PhysR<Real> q = phys_r<Real>(p);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * DTX + tx;
    const int i0 = bx * L::TX + 1, j0 = by * DTY + 1;
    const int j = j0 + ty;
    const int k0 = bz * zchunk + 1;
    const int k1 = min(k0 + zchunk - 1, g.gz);
    const int nplanes = k1 - k0 + 3;  // k0-1 .. k1+1
    const CUtensorMap *mcl = &maps.cl[pin];
    const CUtensorMap *mfs = &maps.fs[pin];
    const unsigned base = ring;

    auto stage = [&](int s) { return smem + s * L::BYTES; };
    auto issue = [&](int pl) {
        const int s = (int)((base + pl) % TS), k = k0 - 1 + pl;
        const bool center = (k >= k0 && k <= k1);
        mbar_expect_tx(&bars[s], L::TX_HALO + (center ? L::TX_CENTER : 0u));
        tma_load_3d(stage(s), mcl, i0 - 1, j0 - 1, k, &bars[s]);
        tma_load_3d(stage(s) + L::CL, mfs, i0 - 1, j0 - 1, k, &bars[s]);
        if (center) {
            tma_load_3d(stage(s) + 2 * L::CL, &maps.ce, i0 + L::LEAD, j0, k, &bars[s]);
            tma_load_3d(stage(s) + 2 * L::CL + L::CE, &maps.gr, i0 + 3, j0, k, &bars[s]);
        }
    };
    auto phase = [&](int pl) { return (unsigned)(((base + pl) / TS) & 1u); };
    // temperature of each plane of the chunk when it depends on z only
    // (direct_temp_calc's isothermal and gradient models in 3D)
    const bool t_per_plane = (p.temp_mode == 0) || (p.temp_mode == 1 && !p.gz_is_one);
    if (tid == 0) sh.abort = 0;
    if (t_per_plane && tid <= k1 - k0) sh.sT[tid] = temp_cell(p, a.d.T, a.d.T32, 0, 1, k0 + tid, ts);
    __syncthreads();
    if (tid == 0)
        for (int pl = 0; pl < TS && pl < nplanes; pl++) issue(pl);
    int issued = min(TS, nplanes);  // same value in every thread

    const Real one_x = (Real)(1 - g.padx), one_y = (Real)(1 - g.pady), one_zp = (Real)(1 - g.padz_hi),
               one_zm = (Real)(1 - g.padz_lo);
    const long long wrow = (long long)g.wpr;
    // plane-invariant per-cell values
    int hh[CPT], hcc[CPT], hgg[CPT];
    bool act[CPT], in_xy[CPT];
    Real omx_p[CPT], omx_m[CPT];
    const bool jrow = j <= g.gy;
    const Real omy_p = j == g.gy ? one_y : (Real)1, omy_m = j == 1 ? one_y : (Real)1;
#pragma unroll
    for (int u = 0; u < CPT; u++) {
        const int i = i0 + tx + DTX * u;
        hh[u] = (ty + 1) * L::BXH + tx + DTX * u + L::HX;
        hcc[u] = ty * L::BXC + tx + DTX * u;
        hgg[u] = ty * L::BXG + tx + DTX * u;
        act[u] = i <= g.gx && jrow;
        in_xy[u] = i > 1 && i < g.gx && j > 1 && j < g.gy;
        omx_p[u] = i == g.gx ? one_x : (Real)1;
        omx_m[u] = i == 1 ? one_x : (Real)1;
    }
    // ring slots of planes t, t+1, t+2 and the phase of slot s2
    int s0 = (int)(base % TS), s1 = (int)((base + 1) % TS), s2 = (int)((base + 2) % TS);
    unsigned ph2 = phase(2);
    long long crow = (long long)k0 * g.sz + (long long)j * g.sy;
    bool alive = true;
    double fsum = 0.0;  // this thread's new fs values, in plane order
    // AM temperature array: each cell's value is loaded one plane ahead, so
    // that its latency overlaps a plane of work
    const bool t_arr = p.temp_mode == 2;
    double Tn[CPT];
    // (the FP32 form keeps it in FP32)
    auto t_load = [&](long long c) -> double {
        return sizeof(Real) == 4 ? (double)__ldg(a.d.T32 + c) : __ldg(a.d.T + c);
    };
#pragma unroll
    for (int u = 0; u < CPT; u++) Tn[u] = (t_arr && act[u]) ? t_load(crow + i0 + tx + DTX * u) : 0.0;
    for (int t = 0; t <= k1 - k0; t++) {
        const int k = k0 + t;
        double Tc[CPT];
#pragma unroll
        for (int u = 0; u < CPT; u++) {
            Tc[u] = Tn[u];
            if (t_arr && act[u] && t < k1 - k0) Tn[u] = t_load(crow + g.sz + i0 + tx + DTX * u);
        }
        // planes t and t+1 completed in earlier iterations
        bool ok = mbar_wait(&bars[s2], ph2);
        if (t == 0) ok &= mbar_wait(&bars[s0], phase(0)) && mbar_wait(&bars[s1], phase(1));
        if (!ok) sh.abort = 1;
        int solid[CPT];
        const Real *cm = (const Real *)stage(s0);
        const Real *cc = (const Real *)stage(s1);
        const Real *cp = (const Real *)stage(s2);
        const Real *fm = (const Real *)(stage(s0) + L::CL);
        const Real *fc = (const Real *)(stage(s1) + L::CL);
        const Real *fp = (const Real *)(stage(s2) + L::CL);
        const Real *sce = (const Real *)(stage(s1) + 2 * L::CL);
        const int *sgr = (const int *)(stage(s1) + 2 * L::CL + L::CE);
        const Real omz_p = k == g.gz ? one_zp : (Real)1, omz_m = k == 1 ? one_zm : (Real)1;
        const bool in_z = k > 1 && k < g.gz;
        const double Tp = t_per_plane ? sh.sT[t] : 0.0;
#pragma unroll
        for (int u = 0; u < CPT; u++) {
            solid[u] = 0;
            if (act[u] && ok) {
                const int h = hh[u];
                const int i = i0 + tx + DTX * u;
                const Real nb_cl[6] = {cc[h + 1], cc[h - 1], cc[h + L::BXH], cc[h - L::BXH], cp[h], cm[h]};
                const Real nb_fs[6] = {fc[h + 1], fc[h - 1], fc[h + L::BXH], fc[h - L::BXH], fp[h], fm[h]};
                const Real one_m[6] = {omx_p[u], omx_m[u], omy_p, omy_m, omz_p, omz_m};
                const long long c = crow + i;
                const Real oce = sce[hcc[u]];
                const int grc = sgr[hgg[u]];
                const double Td = t_per_plane ? Tp : (t_arr ? Tc[u] : temp_cell(p, a.d.T, a.d.T32, c, j, k, ts));
                const bool interior = in_xy[u] && in_z;
                Real cen, cl_new, fs_new;
                int gr_new, br;
                cell_update<Real>(q, p, cc[h], fc[h], nb_cl, nb_fs, one_m, interior, oce, grc, Td, a.d.curv, c,
                                  cen, cl_new, fs_new, gr_new, br, sizeof(Real) == 4 && t_arr);
                if (!in_bounds(ctl, c, g.N)) continue;
                ce[c] = cen;
                clO[c] = cl_new;
                fsO[c] = fs_new;
                if (gr_new != grc) gr[c] = gr_new;
                // growth.c:163-165 (the FP32 form stores ce - Cinit)
                if (sizeof(Real) == 8 ? cen < 0 : cen < -q.cinit) raise_error(ctl, MMS_ERR_NEGATIVE_CE);
                solid[u] = gr_new > 0;
                if (part) fsum += (double)fs_new;
            }
        }
#pragma unroll
        for (int u = 0; u < CPT; u++) {
            const unsigned word = __ballot_sync(FULL_MASK, solid[u]);
            const int w = bx * CPT + u;
            if (tx == 0 && jrow && w < g.wpr) {
                const long long wi = ((long long)k * (g.gy + 2) + j) * wrow + w;
                if (in_bounds(ctl, wi, g.nwords)) a.d.solid_bits[wi] = word;
            }
        }
        __syncthreads();
        if (sh.abort) {
            // a copy did not land within the bound: report, then wait (again
            // bounded) for every copy still in flight before leaving
            if (tid == 0) {
                raise_error(ctl, MMS_ERR_TIMEOUT);
                for (int pl = t; pl < issued; pl++) mbar_wait(&bars[(base + pl) % TS], phase(pl));
            }
            alive = false;
            break;
        }
        if (t + TS < nplanes) {
            if (tid == 0) issue(t + TS);
            issued = t + TS + 1;
        }
        // advance the ring
        s0 = s1;
        s1 = s2;
        s2 = (s2 + 1 == TS) ? 0 : s2 + 1;
        if (s2 == 0) ph2 ^= 1u;
        crow += g.sz;
    }
    ring = base + (unsigned)nplanes;
    if (part && alive) {
        // fixed-order tree: lanes, then the 8 warps
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) fsum += __shfl_down_sync(FULL_MASK, fsum, o);
        if (tx == 0) sh.fsum[ty] = fsum;
        __syncthreads();
        if (tid == 0) {
            double v = 0.0;
#pragma unroll
            for (int w = 0; w < DTY; w++) v += sh.fsum[w];
            part[2 * part_idx] = v;
            part[2 * part_idx + 1] = 0.0;
        }
    }
    return alive;
}

// Two adjacent cells per thread (CPT = 2): thread tx of row ty owns cells
// i = i0 + 2 tx and i + 1.  Each plane it reads the pair and its four x/y
// neighbour pairs of cl and fs as single 8- (FP32) or 16-byte (FP64) words
// of shared memory, the pair above (plane k + 1) likewise, and takes the
// pairs of planes k and k - 1 from registers, rolled up the z-chunk; the x
// neighbours of the two cells are the neighbouring pairs' inner halves.  The
// FP32 form sums the six neighbour terms of both cells with paired FP32
// instructions (each component rounds exactly as the scalar fmaf chain of
// diff_sum); the FP64 form sums each cell in the reference's order.  Cells,
// temperatures and results move as one word per field and pair.  The solid
// bitmask words of the CTA's 64 cells come from two warp OR-reductions.
template <typename Real>
struct Vec2;
template <>
struct Vec2<float> {
    using T = float2;
};
template <>
struct Vec2<double> {
    using T = double2;
};

template <typename Real>
__device__ __forceinline__ typename Vec2<Real>::T vec2(Real x, Real y)
{
    typename Vec2<Real>::T v;
    v.x = x;
    v.y = y;
    return v;
}

// TM, FP32 form only: 1 with an FP32 temperature array (the AM model), whose
// cells take the FP32-temperature update; 2 with a temperature per plane,
// whose difference from the liquidus and range test are formed once per
// plane; 0 otherwise.  Separate instantiations, so that each inner loop
// carries only its own form; all give what fs_update gives.
template <typename Real, int TM = 0>
__device__ __forceinline__ bool stencil_tile_pair(const KernelArgs &a, const TmaMaps &maps, int zchunk, int bx, int by,
                                                  int bz, unsigned char *smem, StencilShared<Depth<Real, 2>::TS> &sh,
                                                  unsigned &ring, double *part = nullptr, long long part_idx = 0)
{
    using L = Stage<Real, 2>;
    using V = typename Vec2<Real>::T;
    constexpr int TS = Depth<Real, 2>::TS;
    Ctl *ctl = a.d.ctl;
    unsigned long long *bars = sh.bars;
    const Geo &g = a.g;
    const Phys &p = a.p;
    const unsigned long long ts = ctl->timestep;
    const int pin = (int)((ts - 1) & 1ULL), pout = (int)(ts & 1ULL);
    Real *__restrict__ clO = (Real *)a.d.cl[pout];
    Real *__restrict__ fsO = (Real *)a.d.fs[pout];
    Real *__restrict__ ce = (Real *)a.d.ce;
    int *__restrict__ gr = a.d.gr;
    const PhysR<Real> q = phys_r<Real>(p);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * DTX + tx;
    const int i0 = bx * L::TX + 1, j0 = by * DTY + 1;
    const int i = i0 + 2 * tx, j = j0 + ty;
    const int k0 = bz * zchunk + 1;
    const int k1 = min(k0 + zchunk - 1, g.gz);
    const int nplanes = k1 - k0 + 3;  // k0-1 .. k1+1
    const CUtensorMap *mcl = &maps.cl[pin];
    const CUtensorMap *mfs = &maps.fs[pin];
    const unsigned base = ring;

    auto stage = [&](int s) { return smem + s * L::BYTES; };
    auto issue = [&](int pl) {
        const int s = (int)((base + pl) % TS), k = k0 - 1 + pl;
        const bool center = (k >= k0 && k <= k1);
        mbar_expect_tx(&bars[s], L::TX_HALO + (center ? L::TX_CENTER : 0u));
        tma_load_3d(stage(s), mcl, i0 - 1, j0 - 1, k, &bars[s]);
        tma_load_3d(stage(s) + L::CL, mfs, i0 - 1, j0 - 1, k, &bars[s]);
        if (center) {
            tma_load_3d(stage(s) + 2 * L::CL, &maps.ce, i0 + L::LEAD, j0, k, &bars[s]);
            tma_load_3d(stage(s) + 2 * L::CL + L::CE, &maps.gr, i0 + 3, j0, k, &bars[s]);
        }
    };
    auto phase = [&](int pl) { return (unsigned)(((base + pl) / TS) & 1u); };
    const bool t_per_plane = (p.temp_mode == 0) || (p.temp_mode == 1 && !p.gz_is_one);
    if (tid == 0) sh.abort = 0;
    if (t_per_plane && tid <= k1 - k0) sh.sT[tid] = temp_cell(p, a.d.T, a.d.T32, 0, 1, k0 + tid, ts);
    __syncthreads();
    if (tid == 0)
        for (int pl = 0; pl < TS && pl < nplanes; pl++) issue(pl);
    int issued = min(TS, nplanes);  // same value in every thread

    const Real one_x = (Real)(1 - g.padx), one_y = (Real)(1 - g.pady), one_zp = (Real)(1 - g.padz_hi),
               one_zm = (Real)(1 - g.padz_lo);
    const long long wrow = (long long)g.wpr;
    const bool jrow = j <= g.gy;
    const bool act0 = i <= g.gx && jrow, act1 = i + 1 <= g.gx && jrow;
    // (1 - mold) of the faces: +x and -x of cell i, +x of cell i + 1 (its -x
    // face is cell i), +y and -y of both
    const Real o0xp = i == g.gx ? one_x : (Real)1, o0xm = i == 1 ? one_x : (Real)1;
    const Real o1xp = i + 1 == g.gx ? one_x : (Real)1;
    const Real omy_p = j == g.gy ? one_y : (Real)1, omy_m = j == 1 ? one_y : (Real)1;
    // the CTA's tile touches a domain face in x or y (uniform over the CTA);
    // elsewhere every (1 - mold) factor is 1 and the (exact) product by it is
    // skipped
    const bool edge_xy = (i0 == 1) || (i0 + L::TX - 1 >= g.gx) || (j0 == 1) || (j0 + DTY - 1 >= g.gy);
    const int hc = (ty + 1) * L::BXH + L::HX + 2 * tx;  // cell i in a cl/fs box
    const int hcc = ty * L::BXC + 2 * tx;                // cell i in a ce/gr box
    int s0 = (int)(base % TS), s1 = (int)((base + 1) % TS), s2 = (int)((base + 2) % TS);
    unsigned ph2 = phase(2);
    long long crow = (long long)k0 * g.sz + (long long)j * g.sy;
    bool alive = true;
    double fsum = 0.0;  // this thread's new fs values, in plane order
    // AM temperature array (FP32 in the FP32 form): the pair's values are
    // loaded two planes ahead, so that their latency overlaps two planes of
    // work
    const bool t_arr = p.temp_mode == 2;
    auto t_load = [&](long long c) -> V {
        if (sizeof(Real) == 4) {
            const float2 v = __ldg((const float2 *)(a.d.T32 + c));
            return vec2<Real>((Real)v.x, (Real)v.y);
        }
        const double2 v = __ldg((const double2 *)(a.d.T + c));
        return vec2<Real>((Real)v.x, (Real)v.y);
    };
    V Tn = vec2<Real>(0, 0), Tnn = Tn;
    if (t_arr && act0) {
        Tn = t_load(crow + i);
        if (k1 > k0) Tnn = t_load(crow + g.sz + i);
    }
    V zm_cl = vec2<Real>(0, 0), zc_cl = zm_cl, zm_fs = zm_cl, zc_fs = zm_cl;
    for (int t = 0; t <= k1 - k0; t++) {
        const int k = k0 + t;
        const Real Tn0 = Tn.x, Tn1 = Tn.y;
        const double T0 = (double)Tn.x, T1 = (double)Tn.y;
        Tn = Tnn;
        if (t_arr && act0 && t + 1 < k1 - k0) Tnn = t_load(crow + 2 * g.sz + i);
        // planes t and t+1 completed in earlier iterations
        bool ok = mbar_wait(&bars[s2], ph2);
        if (t == 0) ok &= mbar_wait(&bars[s0], phase(0)) && mbar_wait(&bars[s1], phase(1));
        if (!ok) sh.abort = 1;
        const Real *cc = (const Real *)stage(s1), *cp = (const Real *)stage(s2);
        const Real *fc = (const Real *)(stage(s1) + L::CL), *fp = (const Real *)(stage(s2) + L::CL);
        const Real *sce = (const Real *)(stage(s1) + 2 * L::CL);
        const int *sgr = (const int *)(stage(s1) + 2 * L::CL + L::CE);
        if (t == 0 && ok) {
            zm_cl = *(const V *)((const Real *)stage(s0) + hc);
            zm_fs = *(const V *)((const Real *)(stage(s0) + L::CL) + hc);
            zc_cl = *(const V *)(cc + hc);
            zc_fs = *(const V *)(fc + hc);
        }
        const Real omz_p = k == g.gz ? one_zp : (Real)1, omz_m = k == 1 ? one_zm : (Real)1;
        const bool edge = edge_xy || k == 1 || k == g.gz;
        V zp_cl = zc_cl, zp_fs = zc_fs;
        int solid0 = 0, solid1 = 0;
        if (act0 && ok) {
            zp_cl = *(const V *)(cp + hc);
            zp_fs = *(const V *)(fp + hc);
            const V lcl = *(const V *)(cc + hc - 2), rcl = *(const V *)(cc + hc + 2);
            const V ucl = *(const V *)(cc + hc + L::BXH), dcl = *(const V *)(cc + hc - L::BXH);
            const V lfs = *(const V *)(fc + hc - 2), rfs = *(const V *)(fc + hc + 2);
            const V ufs = *(const V *)(fc + hc + L::BXH), dfs = *(const V *)(fc + hc - L::BXH);
            const V oce = *(const V *)(sce + hcc);
            const int2 grc = *(const int2 *)(sgr + hcc);
            Real nb0, nb1;
            if (sizeof(Real) == 4) {
                // the neighbour terms of both cells at once: +x, -x, +y, -y, +z, -z
                const float B = 0.5f * ((float)q.rs - (float)q.rl);
                const float2 B2 = make_float2(B, B), rl2 = make_float2((float)q.rl, (float)q.rl);
                const float2 conc = make_float2((float)zc_cl.x, (float)zc_cl.y);
                const float2 nconc = make_float2(-conc.x, -conc.y);
                const float2 A2 = __ffma2_rn(B2, make_float2((float)zc_fs.x, (float)zc_fs.y), rl2);
                const float2 ncl[6] = {make_float2((float)zc_cl.y, (float)rcl.x), make_float2((float)lcl.y, (float)zc_cl.x),
                                       make_float2((float)ucl.x, (float)ucl.y), make_float2((float)dcl.x, (float)dcl.y),
                                       make_float2((float)zp_cl.x, (float)zp_cl.y),
                                       make_float2((float)zm_cl.x, (float)zm_cl.y)};
                const float2 nfs[6] = {make_float2((float)zc_fs.y, (float)rfs.x), make_float2((float)lfs.y, (float)zc_fs.x),
                                       make_float2((float)ufs.x, (float)ufs.y), make_float2((float)dfs.x, (float)dfs.y),
                                       make_float2((float)zp_fs.x, (float)zp_fs.y),
                                       make_float2((float)zm_fs.x, (float)zm_fs.y)};
                const float2 om[6] = {make_float2((float)o0xp, (float)o1xp), make_float2((float)o0xm, 1.f),
                                      make_float2((float)omy_p, (float)omy_p), make_float2((float)omy_m, (float)omy_m),
                                      make_float2((float)omz_p, (float)omz_p), make_float2((float)omz_m, (float)omz_m)};
                float2 acc = make_float2(0.f, 0.f);
#pragma unroll
                for (int n = 0; n < 6; n++) {
                    float2 r = __ffma2_rn(B2, nfs[n], A2);
                    if (edge) r = __fmul2_rn(r, om[n]);
                    acc = __ffma2_rn(r, __fadd2_rn(ncl[n], nconc), acc);
                }
                nb0 = (Real)acc.x;
                nb1 = (Real)acc.y;
            } else {
                const Real c0[6] = {zc_cl.y, lcl.y, ucl.x, dcl.x, zp_cl.x, zm_cl.x};
                const Real f0[6] = {zc_fs.y, lfs.y, ufs.x, dfs.x, zp_fs.x, zm_fs.x};
                const Real m0[6] = {o0xp, o0xm, omy_p, omy_m, omz_p, omz_m};
                const Real c1[6] = {rcl.x, zc_cl.x, ucl.y, dcl.y, zp_cl.y, zm_cl.y};
                const Real f1[6] = {rfs.x, zc_fs.x, ufs.y, dfs.y, zp_fs.y, zm_fs.y};
                const Real m1[6] = {o1xp, (Real)1, omy_p, omy_m, omz_p, omz_m};
                nb0 = diff_sum<Real>(q, zc_cl.x, zc_fs.x, c0, f0, m0, !edge);
                nb1 = diff_sum<Real>(q, zc_cl.y, zc_fs.y, c1, f1, m1, !edge);
            }
            const long long c = crow + i;
            const double Tp = t_per_plane ? sh.sT[t] : 0.0;
            const double Td0 = t_per_plane ? Tp : (t_arr ? T0 : temp_cell(p, a.d.T, a.d.T32, c, j, k, ts));
            Real cen0, cl0, fs0;
            int g0, br0;
            // TM 2: the plane temperature's terms of fs_update's FP32 form
            const float dTp = TM == 2 ? (float)(Tp - p.Tliq) : 0.f;
            const bool offp = TM == 2 && (Tp < 1.0 || Tp > p.Tliq);
            if constexpr (sizeof(Real) == 4 && TM == 1) {
                // the FP32 temperature array straight into the FP32 update
                float dT;
                bool off;
                am_dt(q, (float)Tn0, dT, off);
                fs_update_f32(q, p, zc_cl.x, zc_fs.x, nb0, oce.x, grc.x, dT, off, a.d.curv, c, cen0, cl0, fs0, g0, br0);
            } else if constexpr (sizeof(Real) == 4 && TM == 2) {
                fs_update_f32(q, p, zc_cl.x, zc_fs.x, nb0, oce.x, grc.x, dTp, offp, a.d.curv, c, cen0, cl0, fs0, g0,
                              br0);
            } else {
                fs_update<Real>(q, p, zc_cl.x, zc_fs.x, nb0, oce.x, grc.x, Td0, a.d.curv, c, cen0, cl0, fs0, g0, br0);
            }
            if (sizeof(Real) == 8 ? cen0 < 0 : cen0 < -q.cinit) raise_error(ctl, MMS_ERR_NEGATIVE_CE);
            solid0 = g0 > 0;
            if (part) fsum += (double)fs0;
            if (act1) {
                const double Td1 = t_per_plane ? Tp : (t_arr ? T1 : temp_cell(p, a.d.T, a.d.T32, c + 1, j, k, ts));
                Real cen1, cl1, fs1;
                int g1, br1;
                if constexpr (sizeof(Real) == 4 && TM == 1) {
                    float dT;
                    bool off;
                    am_dt(q, (float)Tn1, dT, off);
                    fs_update_f32(q, p, zc_cl.y, zc_fs.y, nb1, oce.y, grc.y, dT, off, a.d.curv, c + 1, cen1, cl1, fs1,
                                  g1, br1);
                } else if constexpr (sizeof(Real) == 4 && TM == 2) {
                    fs_update_f32(q, p, zc_cl.y, zc_fs.y, nb1, oce.y, grc.y, dTp, offp, a.d.curv, c + 1, cen1, cl1,
                                  fs1, g1, br1);
                } else {
                    fs_update<Real>(q, p, zc_cl.y, zc_fs.y, nb1, oce.y, grc.y, Td1, a.d.curv, c + 1, cen1, cl1, fs1,
                                    g1, br1);
                }
                if (sizeof(Real) == 8 ? cen1 < 0 : cen1 < -q.cinit) raise_error(ctl, MMS_ERR_NEGATIVE_CE);
                solid1 = g1 > 0;
                if (part) fsum += (double)fs1;
                if (in_bounds(ctl, c + 1, g.N)) {
                    *(V *)(ce + c) = vec2<Real>(cen0, cen1);
                    *(V *)(clO + c) = vec2<Real>(cl0, cl1);
                    *(V *)(fsO + c) = vec2<Real>(fs0, fs1);
                    if (g0 != grc.x || g1 != grc.y) *(int2 *)(gr + c) = make_int2(g0, g1);
                }
            } else if (in_bounds(ctl, c, g.N)) {
                // the last interior cell of an odd-length row: cell i + 1 is the halo
                ce[c] = cen0;
                clO[c] = cl0;
                fsO[c] = fs0;
                if (g0 != grc.x) gr[c] = g0;
            }
        }
        // the CTA's 64 cells of row j: bits 2 tx, 2 tx + 1 of words 2 bx (tx <
        // 16) and 2 bx + 1
        const unsigned mine = ((unsigned)solid0 | ((unsigned)solid1 << 1)) << ((2 * tx) & 31);
        const unsigned w0 = __reduce_or_sync(FULL_MASK, tx < 16 ? mine : 0u);
        const unsigned w1 = __reduce_or_sync(FULL_MASK, tx >= 16 ? mine : 0u);
        if (tx == 0 && jrow) {
            const long long wi = ((long long)k * (g.gy + 2) + j) * wrow + 2 * bx;
            if (2 * bx < g.wpr && in_bounds(ctl, wi, g.nwords)) a.d.solid_bits[wi] = w0;
            if (2 * bx + 1 < g.wpr && in_bounds(ctl, wi + 1, g.nwords)) a.d.solid_bits[wi + 1] = w1;
        }
        __syncthreads();
        if (sh.abort) {
            // a copy did not land within the bound: report, then wait (again
            // bounded) for every copy still in flight before leaving
            if (tid == 0) {
                raise_error(ctl, MMS_ERR_TIMEOUT);
                for (int pl = t; pl < issued; pl++) mbar_wait(&bars[(base + pl) % TS], phase(pl));
            }
            alive = false;
            break;
        }
        if (t + TS < nplanes) {
            if (tid == 0) issue(t + TS);
            issued = t + TS + 1;
        }
        // advance the ring and the thread's column
        s0 = s1;
        s1 = s2;
        s2 = (s2 + 1 == TS) ? 0 : s2 + 1;
        if (s2 == 0) ph2 ^= 1u;
        zm_cl = zc_cl;
        zm_fs = zc_fs;
        zc_cl = zp_cl;
        zc_fs = zp_fs;
        crow += g.sz;
    }
    ring = base + (unsigned)nplanes;
    if (part && alive) {
        // fixed-order tree: lanes, then the 8 warps
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) fsum += __shfl_down_sync(FULL_MASK, fsum, o);
        if (tx == 0) sh.fsum[ty] = fsum;
        __syncthreads();
        if (tid == 0) {
            double v = 0.0;
#pragma unroll
            for (int w = 0; w < DTY; w++) v += sh.fsum[w];
            part[2 * part_idx] = v;
            part[2 * part_idx + 1] = 0.0;
        }
    }
    return alive;
}

// The tile of either width.  Two cells per thread: adjacent pairs in the FP32
// form; in the FP64 form two cells 32 apart (stencil_tile), whose scalar
// loads keep the register count within three CTAs per SM (the FP64 pair tile
// needs two CTAs' budget and measured slower, 4.67 vs 4.82 TB/s at 256^3).
template <typename Real, int CPT>
__device__ __forceinline__ bool run_tile(const KernelArgs &a, const TmaMaps &maps, int zchunk, int bx, int by, int bz,
                                         unsigned char *smem, StencilShared<Depth<Real, CPT>::TS> &sh, unsigned &ring,
                                         double *part = nullptr, long long part_idx = 0)
{
    if constexpr (CPT == 2 && sizeof(Real) == 4)
    {
        // the tile's temperature form (the same test as stencil_tile_pair's
        // t_per_plane)
        if (a.p.temp_mode == 2)
            return stencil_tile_pair<Real, 1>(a, maps, zchunk, bx, by, bz, smem, sh, ring, part, part_idx);
        if (a.p.temp_mode == 0 || (a.p.temp_mode == 1 && !a.p.gz_is_one))
            return stencil_tile_pair<Real, 2>(a, maps, zchunk, bx, by, bz, smem, sh, ring, part, part_idx);
        return stencil_tile_pair<Real, 0>(a, maps, zchunk, bx, by, bz, smem, sh, ring, part, part_idx);
    }
    else
        return stencil_tile<Real, CPT>(a, maps, zchunk, bx, by, bz, smem, sh, ring, part, part_idx);
}

// SUMFS: each tile also leaves its sum of the new fraction solid in
// a.d.fs_part (the step a reduction follows; ~3 % slower otherwise).
template <typename Real, int CPT, bool SUMFS>
__global__ void __launch_bounds__(DTX *DTY, (Depth<Real, CPT>::MINB))
    k_diffuse_fs_tma(const __grid_constant__ KernelArgs a, const __grid_constant__ TmaMaps maps, int zchunk)
{
    constexpr int TS = Depth<Real, CPT>::TS;
    if (stalled(a.d.ctl)) return;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) StencilShared<TS> sh;
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        for (int s = 0; s < TS; s++) mbar_init(&sh.bars[s], 1);
        fence_barrier_init();
    }
    unsigned ring = 0;
    run_tile<Real, CPT>(a, maps, zchunk, blockIdx.x, blockIdx.y, blockIdx.z, smem, sh, ring,
                            SUMFS ? a.d.fs_part : nullptr,
                            ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x);
}

// Many independent domains in one persistent launch: every CTA walks the
// concatenated tile space of all domains (tile_begin: the first tile of
// each), copying the domain's kernel arguments to shared memory and
// keeping its ring and barriers from tile to tile.  Domains whose step has
// stalled are skipped.
struct BatchItem {
    TmaMaps maps;          // first: 128-byte aligned in the item array
    KernelArgs a;
    long long tile_begin;
    int tiles_x, tiles_y, zchunk, pad;
};

template <typename Real, int CPT>
__global__ void __launch_bounds__(DTX *DTY, (Depth<Real, CPT>::MINB))
    k_diffuse_fs_batch(const BatchItem *__restrict__ items, int nitems, long long total_tiles)
{
    constexpr int TS = Depth<Real, CPT>::TS;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) StencilShared<TS> sh;
    __shared__ __align__(16) KernelArgs sa;
    __shared__ int s_item;
    const int tid = threadIdx.y * DTX + threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < TS; s++) mbar_init(&sh.bars[s], 1);
        fence_barrier_init();
    }
    unsigned ring = 0;
    int cur = -1;
    for (long long t = blockIdx.x; t < total_tiles; t += gridDim.x) {
        if (tid == 0) {
            int lo = 0, hi = nitems - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) / 2;
                if (items[mid].tile_begin <= t) lo = mid;
                else hi = mid - 1;
            }
            s_item = lo;
        }
        __syncthreads();
        const int d = s_item;
        if (d != cur) {
            const int *src = (const int *)&items[d].a;
            int *dst = (int *)&sa;
            for (int e = tid; e < (int)(sizeof(KernelArgs) / sizeof(int)); e += DTX * DTY) dst[e] = src[e];
            cur = d;
        }
        __syncthreads();
        if (stalled(sa.d.ctl)) continue;
        const BatchItem &it = items[d];
        const long long local = t - it.tile_begin;
        const int bx = (int)(local % it.tiles_x);
        const int by = (int)((local / it.tiles_x) % it.tiles_y);
        const int bz = (int)(local / ((long long)it.tiles_x * it.tiles_y));
        if (!run_tile<Real, CPT>(sa, it.maps, it.zchunk, bx, by, bz, smem, sh, ring)) break;
    }
}

// Plain-load variant (used when the driver cannot encode the TMA
// descriptors, and for recording runs of the adjoint): three halo'd planes
// in a shared ring filled by the threads.  REC: also stores, per cell, the
// branch fs_change took and the curvature it used.
template <typename Real, bool REC>
__global__ void __launch_bounds__(DTX *DTY) k_diffuse_fs(KernelArgs a, int zchunk)
{
    Ctl *ctl = a.d.ctl;
    if (stalled(ctl)) return;
    const Geo &g = a.g;
    const Phys &p = a.p;
    const unsigned long long ts = ctl->timestep;
    const int pin = (int)((ts - 1) & 1ULL), pout = (int)(ts & 1ULL);
    const Real *__restrict__ clI = (const Real *)a.d.cl[pin];
    const Real *__restrict__ fsI = (const Real *)a.d.fs[pin];
    Real *__restrict__ clO = (Real *)a.d.cl[pout];
    Real *__restrict__ fsO = (Real *)a.d.fs[pout];
    Real *__restrict__ ce = (Real *)a.d.ce;
    int *__restrict__ gr = a.d.gr;
    const PhysR<Real> q = phys_r<Real>(p);

    __shared__ Real s_cl[3][DTY + 2][DTX + 2];
    __shared__ Real s_fs[3][DTY + 2][DTX + 2];

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * DTX + tx;
    const int i0 = blockIdx.x * DTX + 1, j0 = blockIdx.y * DTY + 1;
    const int i = i0 + tx, j = j0 + ty;
    const int k0 = blockIdx.z * zchunk + 1;
    const int k1 = min(k0 + zchunk - 1, g.gz);
    const bool active = (i <= g.gx) && (j <= g.gy);
    constexpr int PW = DTX + 2, PH = DTY + 2, PN = PW * PH;

    auto load_plane = [&](int slot, int k) {
        for (int e = tid; e < PN; e += DTX * DTY) {
            int ey = e / PW, ex = e - ey * PW;
            int ii = i0 - 1 + ex, jj = j0 - 1 + ey;
            if (ii <= g.gx + 1 && jj <= g.gy + 1) {
                long long c = (long long)k * g.sz + (long long)jj * g.sy + ii;
                s_cl[slot][ey][ex] = clI[c];
                s_fs[slot][ey][ex] = fsI[c];
            }
        }
    };

    load_plane(0, k0 - 1);
    load_plane(1, k0);
    int sm = 0, sc = 1, sp = 2;
    const Real one_x = (Real)(1 - g.padx), one_y = (Real)(1 - g.pady), one_zp = (Real)(1 - g.padz_hi),
               one_zm = (Real)(1 - g.padz_lo);
    for (int k = k0; k <= k1; k++) {
        load_plane(sp, k + 1);
        __syncthreads();
        int solid = 0;
        if (active) {
            const long long c = (long long)k * g.sz + (long long)j * g.sy + i;
            const int ly = ty + 1, lx = tx + 1;
            const Real nb_cl[6] = {s_cl[sc][ly][lx + 1], s_cl[sc][ly][lx - 1], s_cl[sc][ly + 1][lx],
                                   s_cl[sc][ly - 1][lx], s_cl[sp][ly][lx], s_cl[sm][ly][lx]};
            const Real nb_fs[6] = {s_fs[sc][ly][lx + 1], s_fs[sc][ly][lx - 1], s_fs[sc][ly + 1][lx],
                                   s_fs[sc][ly - 1][lx], s_fs[sp][ly][lx], s_fs[sm][ly][lx]};
            const Real one_m[6] = {i == g.gx ? one_x : (Real)1, i == 1 ? one_x : (Real)1,
                                   j == g.gy ? one_y : (Real)1, j == 1 ? one_y : (Real)1,
                                   k == g.gz ? one_zp : (Real)1, k == 1 ? one_zm : (Real)1};
            const int grc = gr[c];
            const double Td = temp_cell(p, a.d.T, a.d.T32, c, j, k, ts);
            Real cen, cl_new, fs_new;
            int gr_new, br;
            const bool interior = i > 1 && i < g.gx && j > 1 && j < g.gy && k > 1 && k < g.gz;
            cell_update<Real>(q, p, s_cl[sc][ly][lx], s_fs[sc][ly][lx], nb_cl, nb_fs, one_m, interior, ce[c], grc,
                              Td, a.d.curv, c, cen, cl_new, fs_new, gr_new, br, sizeof(Real) == 4 && p.temp_mode == 2);
            ce[c] = cen;
            clO[c] = cl_new;
            fsO[c] = fs_new;
            if (gr_new != grc) gr[c] = gr_new;
            if (REC) {
                // frozen-CA record of this step (adjoint replay)
                const long long slot = (long long)(ts - a.d.rec_t0 - 1);
                if (slot >= 0 && slot < a.d.rec_cap) {
                    a.d.rec_flags[slot * g.N + c] = (unsigned char)br;
                    if (p.tip_curv) a.d.rec_curv[slot * g.N + c] = a.d.curv[c];
                }
            }
            // growth.c:163-165 (the FP32 form stores ce - Cinit)
            if (sizeof(Real) == 8 ? cen < 0 : cen < -q.cinit) raise_error(ctl, MMS_ERR_NEGATIVE_CE);
            solid = gr_new > 0;
        }
        const unsigned word = __ballot_sync(FULL_MASK, solid);
        if (tx == 0 && j <= g.gy)
            a.d.solid_bits[((long long)k * (g.gy + 2) + j) * (long long)g.wpr + blockIdx.x] = word;
        __syncthreads();
        int t = sm;
        sm = sc;
        sc = sp;
        sp = t;
    }
}

// ------------------------------------------------------- interface list
// grow_cell_reduction (growth.c:461-538): a non-mold liquid cell with a
// solid face neighbour (all grain ids are >= 0, so "sum of the six
// neighbours' ids > 0" is "some neighbour solid").  Interior cells are
// never mold in one domain.
constexpr int LIST_NT = 256;

// 32 bits of a bitmask row starting at interior cell x (0-based, x >= -1);
// bits outside the row read as 0 (halo cells are never solid).
__device__ __forceinline__ unsigned row_bits(const unsigned *row, int wpr, long long x)
{
    long long w = (x >= 0) ? (x >> 5) : -1;
    int sh = (int)(x - 32 * w);
    unsigned lo = (w >= 0) ? row[w] : 0u;
    unsigned hi = (w + 1 < wpr) ? row[w + 1] : 0u;
    return sh ? (lo >> sh) | (hi << (32 - sh)) : lo;
}

// A piece is 32 consecutive cells of one emulated rank's local row; pieces
// are numbered in rank-local raster order, so list order = piece order.
// Its list membership bits come straight from the solid bitmask: liquid
// and some face neighbour solid.
struct Piece {
    unsigned bits;
    long long base;  // device index of the piece's first cell
};

__device__ __forceinline__ Piece piece_of(const KernelArgs &a, int r, long long q)
{
    const Geo &g = a.g;
    Piece pc{0u, 0};
    if (q >= g.pieces_per_rank) return pc;
    // pieces of one rank number fewer than 2^31 (sby * sbz * ppr): 32-bit division
    const unsigned qq = (unsigned)q, ppr = (unsigned)g.ppr, sby = (unsigned)g.sby;
    const unsigned lr = qq / ppr;
    const int part = (int)(qq - lr * ppr);
    const unsigned lz = lr / sby;
    const int ly = (int)(lr - lz * sby);
    int rx = r % g.nsbx, ry = (r / g.nsbx) % g.nsby, rz = r / (g.nsbx * g.nsby);
    long long J = (long long)ry * g.sby + ly + 1, K = (long long)rz * g.sbz + lz + 1;
    long long X0 = (long long)rx * g.sbx + 32LL * part;  // 0-based interior x
    int len = min(32, g.sbx - 32 * part);
    const long long wpr = g.wpr, plane = wpr * (g.gy + 2);
    const unsigned *row = a.d.solid_bits + (K * (g.gy + 2) + J) * wpr;
    unsigned S = row_bits(row, g.wpr, X0);
    unsigned nb = row_bits(row, g.wpr, X0 - 1) | row_bits(row, g.wpr, X0 + 1) |
                  row_bits(row + wpr, g.wpr, X0) | row_bits(row - wpr, g.wpr, X0) |
                  row_bits(row + plane, g.wpr, X0) | row_bits(row - plane, g.wpr, X0);
    unsigned bits = ~S & nb;
    if (len < 32) bits &= (1u << len) - 1u;
    pc.bits = bits;
    pc.base = K * g.sz + J * g.sy + X0 + 1;
    return pc;
}

// q / d and q % d for 32-bit q with m = floor(2^32 / d): the estimate
// __umulhi(q, m) is the quotient or one less.
__device__ __forceinline__ unsigned fast_divmod(unsigned q, unsigned d, unsigned m, unsigned &rem)
{
    unsigned k = __umulhi(q, m);
    unsigned r = q - k * d;
    if (r >= d) {
        k++;
        r -= d;
    }
    rem = r;
    return k;
}

// piece_of for subblock rows that start on a bitmask word (sbx a multiple
// of 32): seven aligned words per piece; (rx, ry, rz) is rank r's subblock.
__device__ __forceinline__ Piece piece_aligned(const KernelArgs &a, int rx, int ry, int rz, long long q)
{
    const Geo &g = a.g;
    Piece pc{0u, 0};
    if (q >= g.pieces_per_rank) return pc;
    unsigned part, ly;
    const unsigned lr = fast_divmod((unsigned)q, (unsigned)g.ppr, g.ppr_m, part);
    const unsigned lz = fast_divmod(lr, (unsigned)g.sby, g.sby_m, ly);
    const long long J = (long long)ry * g.sby + ly + 1, K = (long long)rz * g.sbz + lz + 1;
    const long long X0 = (long long)rx * g.sbx + 32LL * part;  // 0-based interior x, a multiple of 32
    const long long wpr = g.wpr, plane = wpr * (g.gy + 2);
    const long long w = X0 >> 5;
    const unsigned *row = a.d.solid_bits + (K * (g.gy + 2) + J) * wpr + w;
    const unsigned C = row[0];
    const unsigned L = (w > 0) ? row[-1] : 0u;
    const unsigned R = (w + 1 < wpr) ? row[1] : 0u;
    const unsigned nb = ((C << 1) | (L >> 31)) | ((C >> 1) | (R << 31)) | row[wpr] | row[-wpr] | row[plane] |
                        row[-plane];
    pc.bits = ~C & nb;  // sbx - 32 part >= 32: all 32 cells belong to the piece
    pc.base = K * g.sz + J * g.sy + X0 + 1;
    return pc;
}

// Status word of a list block for the decoupled look-back: bits 34-63 the
// step (low 30 bits of the timestep, so words of earlier steps never
// match), bits 32-33 the state (1 = own count, 2 = inclusive prefix), bits
// 0-31 the value.
constexpr unsigned long long LS_AGG = 1ULL, LS_PRE = 2ULL;
__device__ __forceinline__ unsigned long long ls_word(unsigned long long tag, unsigned long long state, int v)
{
    return (tag << 34) | (state << 32) | (unsigned)v;
}

// Bounded wait for list block j's status word of this step; returns it,
// or 0 after `polls` polls (0: 2^22, about a second).
__device__ __forceinline__ unsigned long long ls_wait(const unsigned long long *st, long long j,
                                                      unsigned long long tag, unsigned long long want_state,
                                                      unsigned polls)
{
    const unsigned n = polls ? polls : (1u << 22);
    for (unsigned it = 0; it < n; it++) {
        unsigned long long w = *((volatile const unsigned long long *)&st[j]);
        if ((w >> 34) == tag && ((w >> 32) & 3ULL) >= want_state) return w;
        if (it > 32) __nanosleep(128);
    }
    return 0;
}

// grow_cell_reduction in one pass: every block counts its pieces, finds the
// list position of its first entry by looking back over the status words
// of the blocks before it, and writes its entries in piece order.  Blocks
// take their list position from a ticket (reset by k_act each step), so a
// block only ever waits on blocks that started before it.  The last block
// of each emulated rank applies the dc_tmp re-allocation rule of
// capture_octahedra_diffuse (growth.c:642-660): when the rank's list
// outgrows its dc_tmp, the reference replaces it with a zeroed array of
// gindex + 100 entries; here the slots that must read as zero this step are
// recorded (rank_zero_upto) and k_capture clears them.
__device__ __forceinline__ void list_body(const KernelArgs &a, int nblocks)
{
    Ctl *ctl = a.d.ctl;
    if (stalled(ctl)) return;
    constexpr int NI = LIST_PIECES / LIST_NT;
    __shared__ int sh[LIST_NT / 32];
    __shared__ int s_b, s_excl, s_ok;
    const Geo &g = a.g;
    unsigned long long *st = a.d.list_status;
    const unsigned long long tag = ctl->timestep & 0x3fffffffULL;
    if (threadIdx.x == 0) s_b = atomicAdd(&ctl->list_ticket, 1);
    __syncthreads();
    const int b = s_b;
    if (b >= nblocks) {  // the ticket was not reset: never index past the block arrays
        if (threadIdx.x == 0) raise_error(ctl, MMS_ERR_STATE);
        return;
    }
    const int r = (int)(b / g.blocks_per_rank);
    const long long q0 = (b % g.blocks_per_rank) * (long long)LIST_PIECES;
    // piece it of this thread: q0 + it * LIST_NT + thread (neighbouring
    // threads read neighbouring bitmask words)
    unsigned bits[NI];
    long long base[NI];
    int ex[NI], tot[NI], agg = 0;
    const bool aligned = (g.sbx & 31) == 0;
    const int rx = r % g.nsbx, ry = (r / g.nsbx) % g.nsby, rz = r / (g.nsbx * g.nsby);
#pragma unroll
    for (int it = 0; it < NI; it++) {
        const long long q = q0 + it * LIST_NT + threadIdx.x;
        const Piece pc = aligned ? piece_aligned(a, rx, ry, rz, q) : piece_of(a, r, q);
        bits[it] = pc.bits;
        base[it] = pc.base;
    }
#pragma unroll
    for (int it = 0; it < NI; it++) {
        ex[it] = block_exclusive_scan<LIST_NT>(__popc(bits[it]), tot[it], sh);
        agg += tot[it];
    }
    // warp 0: decoupled look-back, 32 predecessors per round
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        int excl = 0, ok = 1;
        const unsigned polls = ctl->wait_polls;
        // test hook: a held block publishes nothing (its successor's wait runs out)
        const bool held = ctl->hold_list_block == b + 1;
        if (b > 0) {
            if (lane == 0 && !held) *((volatile unsigned long long *)&st[b]) = ls_word(tag, LS_AGG, agg);
            long long j0 = b - 1;
            while (true) {
                const long long j = j0 - lane;
                unsigned long long w = ls_word(tag, LS_PRE, 0);  // before block 0: prefix 0
                if (j >= 0) w = ls_wait(st, j, tag, LS_AGG, polls);
                const int bad = __any_sync(FULL_MASK, w == 0);
                if (bad) {
                    ok = 0;
                    break;
                }
                const unsigned pre = __ballot_sync(FULL_MASK, ((w >> 32) & 3ULL) == LS_PRE);
                // nearest predecessor holding its inclusive prefix: the lowest lane
                const int stop = pre ? __ffs(pre) - 1 : 31;
                int v = (lane <= stop) ? (int)(w & 0xffffffffULL) : 0;
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
                excl += v;
                if (pre) break;
                j0 -= 32;
            }
        }
        if (lane == 0) {
            a.d.blk_off[b] = excl;
            __threadfence();
            if (!held) *((volatile unsigned long long *)&st[b]) = ls_word(tag, LS_PRE, excl + agg);
            const long long first = (long long)r * g.blocks_per_rank;
            if (ok && b == first + g.blocks_per_rank - 1) {
                // last block of the rank: its list length and dc_tmp bookkeeping
                int start = excl;
                if (b != first) {
                    if (ls_wait(st, first, tag, LS_PRE, polls)) {
                        __threadfence();
                        start = *((volatile const int *)&a.d.blk_off[first]);
                    } else {
                        ok = 0;
                    }
                }
                const int gindex = excl + agg - start;
                a.d.rank_gindex[r] = gindex;
                const int size = a.d.rank_dcsize[r];
                if (gindex > size) {
                    a.d.rank_zero_upto[r] = size;
                    a.d.rank_dcsize[r] = gindex + 100;
                } else {
                    a.d.rank_zero_upto[r] = 0;
                }
            }
            if (b == nblocks - 1) ctl->list_total = excl + agg;
            if (!ok) raise_error(ctl, MMS_ERR_TIMEOUT);
            s_excl = excl;
            s_ok = ok;
        }
    }
    __syncthreads();
    if (!s_ok) return;
    int pos = s_excl;
#pragma unroll
    for (int it = 0; it < NI; it++) {
        int p0 = pos + ex[it];
        pos += tot[it];
        unsigned m = bits[it];
        while (m) {
            const int bit = __ffs(m) - 1;
            m &= m - 1;
            if (in_bounds(ctl, p0, (long long)g.nranks * g.sbcells) && in_bounds(ctl, base[it] + bit, g.N))
                a.d.list_cell[p0] = base[it] + bit;
            p0++;
        }
    }
}

__global__ void __launch_bounds__(LIST_NT) k_list(KernelArgs a, int nblocks)
{
    list_body(a, nblocks);
}

// capture_octahedra_diffuse, INDEX_SEP branch (growth.c:664-794), for the
// list cell c, with grow_octahedra's half diagonal (growth.c:372-403)
// evaluated for the solid neighbour on demand.  Returns the capturing
// grain id (0 = not captured) and the new octahedron centre.
//
// The pre-capture grain ids (ogr) of interior neighbours are read through
// the solid bitmask (bit set <=> gr > 0 after fs_change), so that ids
// written by captures of the same launch are never mistaken for them; the
// gr of a solid cell, and of a halo cell, is not written during capture.
template <typename Real>
__device__ __forceinline__ int capture_cell(const KernelArgs &a, const Real *fs, long long c, long long I,
                                            long long J, long long K, Dc3 &out)
{
    const Geo &g = a.g;
    const Phys &p = a.p;
    const int *gr = a.d.gr;
    const Dc3 *dc = a.d.dc;
    // neighbour order +x, +y, -x, -y, +z, -z (growth.c:604-610, 674-677)
    const long long ndxs[6] = {c + 1, c + g.sy, c - 1, c - g.sy, c + g.sz, c - g.sz};
    const int nnx[6] = {1, 0, -1, 0, 0, 0}, nny[6] = {0, 1, 0, -1, 0, 0}, nnz[6] = {0, 0, 0, 0, 1, -1};
    int found = -1, gid = 0, fx = 0, fy = 0, fz = 0;
    double g00 = 0, g10 = 0, g20 = 0, g01 = 0, g11 = 0, g21 = 0, g02 = 0, g12 = 0, g22 = 0;
    double dx = 0, dy = 0, dz = 0, dn = 0;
    Dc3 dcn{0, 0, 0};
    // the six neighbours' pre-capture grain ids, their loads issued
    // together: an interior neighbour counts only if its solid bit is set
    // (a liquid neighbour's gr may be changing under a concurrent capture
    // and is then discarded); a halo neighbour's gr is never written here
    int ids[6];
#pragma unroll
    for (int n = 0; n < 6; n++) {
        const long long In = I + nnx[n], Jn = J + nny[n], Kn = K + nnz[n];
        const bool inside = In >= 1 && In <= g.gx && Jn >= 1 && Jn <= g.gy && Kn >= 1 && Kn <= g.gz;
        unsigned w = 1u;
        if (inside) w = a.d.solid_bits[(Kn * (g.gy + 2) + Jn) * (long long)g.wpr + ((In - 1) >> 5)] >> ((In - 1) & 31);
        const int gv = *((volatile const int *)&gr[ndxs[n]]);
        ids[n] = (w & 1u) ? gv : 0;
    }
#pragma unroll
    for (int n = 0; n < 6; n++) {
        long long ndx = ndxs[n];
        int id = ids[n];
        if (id > 0 && (unsigned long long)id < p.max_grains) {
            const double *R = a.d.grain_rot + 9 * (long long)id;
            g00 = R[0]; g01 = R[1]; g02 = R[2];
            g10 = R[3]; g11 = R[4]; g12 = R[5];
            g20 = R[6]; g21 = R[7]; g22 = R[8];
            dcn = dc[ndx];
            double rx0 = 0.0 - dcn.x, ry0 = 0.0 - dcn.y, rz0 = 0.0 - dcn.z;
            double gx0 = g00 * rx0 + g10 * ry0 + g20 * rz0;
            double gy0 = g01 * rx0 + g11 * ry0 + g21 * rz0;
            double gz0 = g02 * rx0 + g12 * ry0 + g22 * rz0;
            double ds1 = fabs(gx0) + fabs(gy0) + fabs(gz0);
            ds1 = (ds1 < 1.5) ? ds1 : 1.5;
            dn = ds1 + (double)fs[ndx] * p.fsgrow;
            double rx1 = -1.0 * nnx[n] - dcn.x;
            double ry1 = -1.0 * nny[n] - dcn.y;
            double rz1 = -1.0 * nnz[n] - dcn.z;
            dx = g00 * rx1 + g10 * ry1 + g20 * rz1;
            dy = g01 * rx1 + g11 * ry1 + g21 * rz1;
            dz = g02 * rx1 + g12 * ry1 + g22 * rz1;
            double dfs = dn - (fabs(dx) + fabs(dy) + fabs(dz));
            if (dfs > 0) {
                found = n;
                fx = nnx[n];
                fy = nny[n];
                fz = nnz[n];
                gid = id;
                break;
            }
        }
    }
    if (found < 0) return 0;
    double ncx = 0., ncz = 0., ncy = 0.;
    double ncd = (dn < 1.0) ? dn : 1.0;
    double dd = dn - ncd;
    if (dx + dy >= 0 && dx - dy > 0 && dx + dz > 0 && dx - dz >= 0) ncx = dd;
    else if (dx + dy <= 0 && dx - dy < 0 && dx + dz < 0 && dx - dz <= 0) ncx = -1. * dd;
    else if (dy + dx > 0 && dy - dx >= 0 && dy + dz >= 0 && dy - dz > 0) ncy = dd;
    else if (dy + dx < 0 && dy - dx <= 0 && dy + dz <= 0 && dy - dz < 0) ncy = -1. * dd;
    else if (dz + dx >= 0 && dz - dx > 0 && dz + dy > 0 && dz - dy >= 0) ncz = dd;
    else ncz = -1. * dd;
    out.x = dcn.x + (double)fx + g00 * ncx + g01 * ncy + g02 * ncz;
    out.y = dcn.y + (double)fy + g10 * ncx + g11 * ncy + g12 * ncz;
    out.z = dcn.z + (double)fz + g20 * ncx + g21 * ncy + g22 * ncz;
    return gid;
}

// Captures every list entry and commits it at once (grid-stride over the
// whole list, so the work is balanced however the interface is
// distributed): dc_tmp slot of a captured entry, then the reference's
// copy-back dc[cell] = dc_tmp[slot] for every entry, captured or not
// (growth.c:789, 797-807), and the captured grain id.
template <typename Real>
__device__ __forceinline__ void capture_body(const KernelArgs &a, int bid, int nb)
{
    const Ctl *ctl = a.d.ctl;
    if (stalled(ctl)) return;
    const Geo &g = a.g;
    const int total = ctl->list_total;
    const Real *fs = (const Real *)a.d.fs[(int)(ctl->timestep & 1ULL)];
    Ctl *ctl_w = a.d.ctl;
    for (long long e = bid * (long long)LIST_NT + threadIdx.x; e < total; e += (long long)nb * LIST_NT) {
        if (!in_bounds(ctl_w, e, (long long)g.nranks * g.sbcells)) break;
        const long long c = a.d.list_cell[e];
        if (!in_bounds(ctl_w, c, g.N)) continue;
        long long K, J, I;
        if (g.N < 0x7fffffffLL) {  // 32-bit division when every index fits
            const unsigned cu = (unsigned)c, szu = (unsigned)g.sz, syu = (unsigned)g.sy;
            const unsigned Ku = cu / szu, rem = cu - Ku * szu, Ju = rem / syu;
            K = Ku;
            J = Ju;
            I = rem - Ju * syu;
        } else {
            K = c / g.sz;
            J = (c - K * g.sz) / g.sy;
            I = c - K * g.sz - J * g.sy;
        }
        int r = 0;
        if (g.nranks > 1) {
            const int rx = (int)((I - 1) / g.sbx), ry = (int)((J - 1) / g.sby), rz = (int)((K - 1) / g.sbz);
            r = rx + ry * g.nsbx + rz * g.nsbx * g.nsby;
        }
        if (!in_bounds(ctl_w, I - 1, g.gx) || !in_bounds(ctl_w, J - 1, g.gy) || !in_bounds(ctl_w, K - 1, g.gz) ||
            !in_bounds(ctl_w, r, g.nranks))
            continue;
        const int rank_start = a.d.blk_off[(long long)r * g.blocks_per_rank];
        const long long sl = e - rank_start + 1;
        if (!in_bounds(ctl_w, a.d.rank_dcbase[r] + sl, (long long)g.nranks * (g.sbcells + 101))) continue;
        Dc3 *slot = a.d.dc_tmp + a.d.rank_dcbase[r] + sl;
        Dc3 out;
        const int gid = capture_cell<Real>(a, fs, c, I, J, K, out);
        if (gid) {
            *slot = out;
            a.d.dc[c] = out;
            a.d.gr[c] = gid;
        } else if (sl <= a.d.rank_zero_upto[r]) {
            // slot of a dc_tmp the reference re-allocated zeroed this step
            *slot = Dc3{0.0, 0.0, 0.0};
            a.d.dc[c] = Dc3{0.0, 0.0, 0.0};
        } else {
            a.d.dc[c] = *slot;
        }
        a.d.list_gid[e] = gid;
    }
}

template <typename Real>
__global__ void __launch_bounds__(LIST_NT, 3) k_capture(KernelArgs a)
{
    capture_body<Real>(a, blockIdx.x, gridDim.x);
}

// The small kernels of a step over many domains, one launch each: block b
// belongs to the domain d with begin[d] <= b < begin[d + 1] (begin: prefix
// sums of the domains' block counts), copies that domain's kernel arguments
// to shared memory and runs the single-domain body with its local block.
__device__ __forceinline__ int batch_find(const int *__restrict__ begin, int n, int b)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (begin[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <int NT>
__device__ __forceinline__ int batch_enter(const void *items, size_t stride, const int *begin, int n,
                                           KernelArgs &sa, int &local)
{
    __shared__ int s_d;
    if (threadIdx.x == 0) s_d = batch_find(begin, n, (int)blockIdx.x);
    __syncthreads();
    const int d = s_d;
    const int *src = (const int *)((const unsigned char *)items + stride * (size_t)d);
    int *dst = (int *)&sa;
    for (int e = threadIdx.x; e < (int)(sizeof(KernelArgs) / sizeof(int)); e += NT) dst[e] = src[e];
    __syncthreads();
    local = (int)blockIdx.x - begin[d];
    return d;
}

template <typename Real>
__global__ void __launch_bounds__(NUC_NT) k_nuc_batch(const void *items, size_t stride, const int *begin, int n)
{
    __shared__ __align__(16) KernelArgs sa;
    int local;
    batch_enter<NUC_NT>(items, stride, begin, n, sa, local);
    nuc_body<Real>(sa, local);
}

__global__ void __launch_bounds__(ACT_NT) k_act_batch(const void *items, size_t stride, const int *begin, int n)
{
    __shared__ __align__(16) KernelArgs sa;
    int local;
    batch_enter<ACT_NT>(items, stride, begin, n, sa, local);
    act_body<ACT_NT>(sa, sa.d.act_scratch);
}

__global__ void __launch_bounds__(LIST_NT) k_list_batch(const void *items, size_t stride, const int *begin, int n)
{
    __shared__ __align__(16) KernelArgs sa;
    int local;
    const int d = batch_enter<LIST_NT>(items, stride, begin, n, sa, local);
    list_body(sa, begin[d + 1] - begin[d]);
}

template <typename Real>
__global__ void __launch_bounds__(LIST_NT) k_capture_batch(const void *items, size_t stride, const int *begin, int n)
{
    __shared__ __align__(16) KernelArgs sa;
    int local;
    const int d = batch_enter<LIST_NT>(items, stride, begin, n, sa, local);
    capture_body<Real>(sa, local, begin[d + 1] - begin[d]);
}


// ------------------------------------------------------------ reductions
constexpr int RED_NT = 256;
// Per-block partial sums over interior cells of min(1, fs) (reduce_fs,
// growth.c:541-566) or of ce.  A warp per interior row at a time: the lanes
// load the row's 16-byte vectors from interior cell 1 on (the field layout
// puts cell 1 of every row on a 16-byte boundary; see the stencil's
// alignment note), and the tail (after the last whole vector) one element
// per lane.  Each
// lane adds its values plainly and enters the row's total into its running
// sum with compensation (TwoSum).  A warp issues every load of a row before
// adding (four or more 16-byte loads per lane in flight).
template <typename Real>
__global__ void __launch_bounds__(RED_NT) k_reduce(KernelArgs a, int what, double *partial)
{
    typedef typename std::conditional<sizeof(Real) == 8, double2, float4>::type V;
    constexpr int VEC = 16 / (int)sizeof(Real);
    const Ctl *ctl = a.d.ctl;
    const Geo &g = a.g;
    const int cur = (int)(ctl->timestep & 1ULL);
    const Real *f = (what == MMS_REDUCE_CE_SUM) ? (const Real *)a.d.ce : (const Real *)a.d.fs[cur];
    const bool cap = what != MMS_REDUCE_CE_SUM;
    const unsigned rows = (unsigned)((long long)g.gy * g.gz);  // fewer than 2^32
    const int lane = threadIdx.x & 31;
    const unsigned warp = (blockIdx.x * RED_NT + threadIdx.x) >> 5, nwarps = (gridDim.x * RED_NT) >> 5;
    const int gx = g.gx;
    const int nfull = gx / VEC;  // vectors covering [1, 1 + VEC nfull)
    const int tail0 = 1 + VEC * nfull, ntail = gx - VEC * nfull;
    // this lane's tail element (0: none)
    const int lone = lane < ntail ? tail0 + lane : 0;
    const unsigned gy = (unsigned)g.gy, gy_m = gy <= 1 ? 0xffffffffu : (unsigned)((1ULL << 32) / gy);
    auto val = [&](Real v) -> double { return (double)((cap && (Real)1 < v) ? (Real)1 : v); };
    double s = 0.0, comp = 0.0;
    // units of work: (row, chunk of up to 128 vectors); a warp walks its
    // rows' units in order with the next unit's loads in flight while it
    // adds the current one (two register buffers, used in turn)
    const int nchunks = max(1, (nfull + 127) / 128);
    struct Buf {
        V x[4];
        Real lone;
    };
    auto load = [&](unsigned r, int c, Buf &b) {
        unsigned jj;
        const unsigned kk = fast_divmod(r, gy, gy_m, jj);
        const Real *row = f + (long long)(kk + 1) * g.sz + (long long)(jj + 1) * g.sy;
        const V *vrow = (const V *)(row + 1);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int p = 128 * c + lane + 32 * k;
            if (p < nfull) b.x[k] = __ldg(vrow + p);
            else std::memset(&b.x[k], 0, sizeof(V));
        }
        b.lone = (c == 0 && lone) ? __ldg(row + lone) : (Real)0;
    };
    auto add_unit = [&](const Buf &b) {
        const Real *e0 = (const Real *)&b.x[0], *e1 = (const Real *)&b.x[1], *e2 = (const Real *)&b.x[2],
                   *e3 = (const Real *)&b.x[3];
        double acc = val(b.lone);
#pragma unroll
        for (int e = 0; e < VEC; e++) acc += (val(e0[e]) + val(e1[e])) + (val(e2[e]) + val(e3[e]));
        const double t = s + acc, bp = t - s;  // TwoSum
        comp += (s - (t - bp)) + (acc - bp);
        s = t;
    };
    unsigned r = warp;
    int c = 0;
    Buf A, B;
    if (r < rows) load(r, c, A);
    // one unit: start loading the next into nb, then add cb
    auto unit = [&](Buf &cb, Buf &nb) -> bool {
        int cn = c + 1;
        unsigned rn = r;
        if (cn == nchunks) {
            cn = 0;
            rn = r + nwarps;
        }
        const bool more = rn < rows;
        if (more) load(rn, cn, nb);
        add_unit(cb);
        r = rn;
        c = cn;
        return more;
    };
    if (r < rows)
        while (unit(A, B) && unit(B, A)) {
        }
    __shared__ double ss[RED_NT], sc[RED_NT];
    ss[threadIdx.x] = s;
    sc[threadIdx.x] = comp;
    __syncthreads();
    for (int w = RED_NT / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            double x = ss[threadIdx.x + w];
            double t = ss[threadIdx.x] + x;
            double bp = t - ss[threadIdx.x];
            sc[threadIdx.x] += sc[threadIdx.x + w] + ((ss[threadIdx.x] - (t - bp)) + (x - bp));
            ss[threadIdx.x] = t;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = ss[0];
        partial[2 * blockIdx.x + 1] = sc[0];
    }
}

// d for every cell (grow_octahedra semantics; 0 where no grain grows)
template <typename Real>
__global__ void k_compute_d(KernelArgs a, double *out)
{
    const Ctl *ctl = a.d.ctl;
    const Geo &g = a.g;
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= g.N) return;
    const Real *fs = (const Real *)a.d.fs[(int)(ctl->timestep & 1ULL)];
    int id = a.d.gr[c];
    double d = 0.0;
    long long K = c / g.sz, J = (c % g.sz) / g.sy, I = c % g.sy;
    bool interior = I >= 1 && I <= g.gx && J >= 1 && J <= g.gy && K >= 1 && K <= g.gz;
    if (interior && id > 0 && (unsigned long long)id < a.p.max_grains) {
        const double *R = a.d.grain_rot + 9 * (long long)id;
        Dc3 v = a.d.dc[c];
        double rx0 = 0.0 - v.x, ry0 = 0.0 - v.y, rz0 = 0.0 - v.z;
        double gx0 = R[0] * rx0 + R[3] * ry0 + R[6] * rz0;
        double gy0 = R[1] * rx0 + R[4] * ry0 + R[7] * rz0;
        double gz0 = R[2] * rx0 + R[5] * ry0 + R[8] * rz0;
        double ds1 = fabs(gx0) + fabs(gy0) + fabs(gz0);
        ds1 = (ds1 < 1.5) ? ds1 : 1.5;
        d = ds1 + (double)fs[c] * a.p.fsgrow;
    }
    out[c] = d;
}

__global__ void k_fill_temperature(KernelArgs a, double *out)
{
    const Ctl *ctl = a.d.ctl;
    const Geo &g = a.g;
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= g.N) return;
    long long K = c / g.sz, J = (c % g.sz) / g.sy;
    out[c] = temp_cell(a.p, a.d.T, a.d.T32, c, J, K, ctl->timestep);
}
// Zero the entries of cells captured by the last step (list cells whose
// capture produced a grain id): turns gr into the reference's ogr, and
// limits d to cells that were solid at the growth step.
template <typename T>
__global__ void k_mask_captured(KernelArgs a, T *out)
{
    const Ctl *ctl = a.d.ctl;
    const int total = ctl->list_total;
    for (long long pos = blockIdx.x * (long long)blockDim.x + threadIdx.x; pos < total;
         pos += (long long)gridDim.x * blockDim.x)
        if (a.d.list_gid[pos]) out[a.d.list_cell[pos]] = (T)0;
}

int launch_mask_captured(const KernelArgs &a, void *dev, int is_double, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (is_double) k_mask_captured<double><<<148 * 4, 256, 0, st>>>(a, (double *)dev);
    else k_mask_captured<int><<<148 * 4, 256, 0, st>>>(a, (int *)dev);
    return 1;
}

// Conversion between the stored precision and FP64 host buffers.
template <typename Real>
__global__ void k_convert(KernelArgs a, int field, int to_device, double *buf)
{
    const Ctl *ctl = a.d.ctl;
    const Geo &g = a.g;
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= g.N) return;
    const int cur = (int)(ctl->timestep & 1ULL);
    Real *f = nullptr, *f2 = nullptr;
    if (field == MMS_FIELD_CE) f = (Real *)a.d.ce;
    else if (field == MMS_FIELD_CL) f = (Real *)a.d.cl[cur], f2 = (Real *)a.d.cl[cur ^ 1];
    else f = (Real *)a.d.fs[cur], f2 = (Real *)a.d.fs[cur ^ 1];
    // the FP32 form stores ce and cl as deviations from Cinit
    const double off = (sizeof(Real) == 4 && field != MMS_FIELD_FS) ? a.p.cinit : 0.0;
    if (to_device) {
        f[c] = (Real)(buf[c] - off);
        if (f2) f2[c] = (Real)(buf[c] - off);
    } else {
        buf[c] = (double)f[c] + off;
    }
}

// k_convert between a field and FP64 values in the reference's halo'd
// layout (ref, row length gx + 2), one block per row of cells at a time.
template <typename Real>
__global__ void k_convert_ref(KernelArgs a, int field, int to_device, double *ref)
{
    const Ctl *ctl = a.d.ctl;
    const Geo &g = a.g;
    const int cur = (int)(ctl->timestep & 1ULL);
    Real *f = nullptr, *f2 = nullptr;
    if (field == MMS_FIELD_CE) f = (Real *)a.d.ce;
    else if (field == MMS_FIELD_CL) f = (Real *)a.d.cl[cur], f2 = (Real *)a.d.cl[cur ^ 1];
    else f = (Real *)a.d.fs[cur], f2 = (Real *)a.d.fs[cur ^ 1];
    const double off = (sizeof(Real) == 4 && field != MMS_FIELD_FS) ? a.p.cinit : 0.0;
    const long long rows = (long long)(g.gy + 2) * (g.gz + 2);
    for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
        Real *fr = f + r * g.P, *fr2 = f2 ? f2 + r * g.P : nullptr;
        double *rr = ref + r * g.rsy;
        for (int i = threadIdx.x; i < g.rsy; i += blockDim.x) {
            if (to_device) {
                const Real v = (Real)(rr[i] - off);
                fr[i] = v;
                if (fr2) fr2[i] = v;
            } else {
                rr[i] = (double)fr[i] + off;
            }
        }
    }
}

// ---------------------------------------------------------------- launch
static int pick_zchunk(const Geo &g, int tile_x)
{
    long long tiles = (long long)((g.gx + tile_x - 1) / tile_x) * ((g.gy + DTY - 1) / DTY);
    // aim for >= 4 CTAs per SM on 148 SMs, chunks of at most 32 planes
    long long want = 148LL * 4;
    int zc = (int)((tiles * g.gz) / want);
    if (zc < 4) zc = 4;
    if (zc > 32) zc = 32;
    if (zc > g.gz) zc = g.gz;
    return zc;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn()
{
    // looked up once, thread-safely (a static initialised by a call), so a
    // context created on another thread meanwhile never sees a half-done
    // lookup and falls back to the plain-load stencil
    static const EncodeTiledFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return (EncodeTiledFn)p;
        return (EncodeTiledFn) nullptr;
    }();
    return fn;
}

// A field as a 3D tensor map with x extent gx + 2 + lead, starting lead =
// 16 / es - 1 elements before the field (at the 16-byte boundary the field's
// allocation keeps there; see the stencil's alignment note).  False when the
// field is not laid out so, or the encoder refuses.
static bool encode3d(CUtensorMap *m, CUtensorMapDataType dt, int es, void *field, const Geo &g, int bx, int by)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    const int lead = 16 / es - 1;
    char *base = (char *)field - (long long)lead * es;
    if (((unsigned long long)base & 15ULL) != 0 || g.P < g.gx + 2 + lead) return false;
    cuuint64_t dims[3] = {(cuuint64_t)(g.gx + 2 + lead), (cuuint64_t)(g.gy + 2), (cuuint64_t)(g.gz + 2)};
    cuuint64_t strides[2] = {(cuuint64_t)(g.P * es), (cuuint64_t)(g.P * (g.gy + 2) * es)};
    cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    return fn(m, dt, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The FP32 temperature field as the target of tensor stores of the AM
// contraction's epilogue (am_tc.cu): x extent gx + 1 + lead, so that a box
// reaching past the last interior cell leaves the right halo column
// untouched; boxes of bx x by x 1.  False when the encoder refuses or the
// field is not laid out with its lead.
bool encode_t32_store(void *map, const KernelArgs &a, int bx, int by)
{
    EncodeTiledFn fn = encode_fn();
    const Geo &g = a.g;
    if (!fn || !a.d.T32) return false;
    const int es = 4, lead = 16 / es - 1;
    char *base = (char *)a.d.T32 - (long long)lead * es;
    if (((unsigned long long)base & 15ULL) != 0 || g.P < g.gx + 2 + lead) return false;
    cuuint64_t dims[3] = {(cuuint64_t)(g.gx + 1 + lead), (cuuint64_t)(g.gy + 2), (cuuint64_t)(g.gz + 2)};
    cuuint64_t strides[2] = {(cuuint64_t)(g.P * es), (cuuint64_t)(g.P * (g.gy + 2) * es)};
    cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    return fn((CUtensorMap *)map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename Real, int CPT>
static int make_tma_t(const KernelArgs &a, TmaHolder &out)
{
    static_assert(sizeof(TmaMaps) <= sizeof(out.bytes), "TMA holder too small");
    using L = Stage<Real, CPT>;
    TmaMaps m;
    std::memset(&m, 0, sizeof m);
    const CUtensorMapDataType dt = sizeof(Real) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const int es = (int)sizeof(Real);
    bool ok = true;
    for (int b = 0; b < 2; b++) {
        ok &= encode3d(&m.cl[b], dt, es, a.d.cl[b], a.g, L::BXH, DTY + 2);
        ok &= encode3d(&m.fs[b], dt, es, a.d.fs[b], a.g, L::BXH, DTY + 2);
    }
    ok &= encode3d(&m.ce, dt, es, a.d.ce, a.g, L::BXC, DTY);
    ok &= encode3d(&m.gr, CU_TENSOR_MAP_DATA_TYPE_INT32, 4, a.d.gr, a.g, L::BXG, DTY);
    if (CPT == 2 && a.p.temp_mode == 2) {
        // the pair tile reads the temperature array in pairs too
        const void *T = sizeof(Real) == 4 ? (const void *)a.d.T32 : (const void *)a.d.T;
        ok &= T && (((unsigned long long)T + sizeof(Real)) & 15ULL) == 0;
    }
    std::memcpy(out.bytes, &m, sizeof m);
    out.ok = ok ? 1 : 0;
    if (ok) {
        cudaFuncSetAttribute(k_diffuse_fs_tma<Real, CPT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             Depth<Real, CPT>::TS * L::BYTES);
        cudaFuncSetAttribute(k_diffuse_fs_tma<Real, CPT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             Depth<Real, CPT>::TS * L::BYTES);
    }
    return out.ok;
}

int make_tma(const KernelArgs &a, int precision, TmaHolder &out)
{
    if (out.cpt != 1 && out.cpt != 2) out.cpt = 1;
    if (precision == MMS_PREC_F32)
        return out.cpt == 2 ? make_tma_t<float, 2>(a, out) : make_tma_t<float, 1>(a, out);
    return out.cpt == 2 ? make_tma_t<double, 2>(a, out) : make_tma_t<double, 1>(a, out);
}

#define PROF_BEGIN(id) \
    if (prof) prof->begin(id, st)
#define PROF_END(id) \
    if (prof) prof->end(id, st)

template <typename Real>
static void launch_stencil_t(const KernelArgs &a, const TmaHolder &tma, cudaStream_t st, bool sumfs = false)
{
    const Geo &g = a.g;
    const int cpt = (tma.ok && tma.cpt == 2) ? 2 : 1;
    const int tile_x = DTX * cpt;
    int zc = tma.zc > 0 ? (tma.zc < g.gz ? tma.zc : g.gz) : pick_zchunk(g, tile_x);
    if (zc > 64) zc = 64;  // sT holds 64 planes
    dim3 grid((g.gx + tile_x - 1) / tile_x, (g.gy + DTY - 1) / DTY, (g.gz + zc - 1) / zc);
    if (a.d.rec_flags) {
        // recording run: plain-load variant with 32-wide tiles
        const int zr = pick_zchunk(g, DTX);
        dim3 gr((g.gx + DTX - 1) / DTX, (g.gy + DTY - 1) / DTY, (g.gz + zr - 1) / zr);
        k_diffuse_fs<Real, true><<<gr, dim3(DTX, DTY), 0, st>>>(a, zr);
    } else if (tma.ok) {
        TmaMaps maps;
        std::memcpy(&maps, tma.bytes, sizeof maps);
        const dim3 blk(DTX, DTY);
        const int b2 = Depth<Real, 2>::TS * Stage<Real, 2>::BYTES, b1 = Depth<Real, 1>::TS * Stage<Real, 1>::BYTES;
        if (cpt == 2 && sumfs) k_diffuse_fs_tma<Real, 2, true><<<grid, blk, b2, st>>>(a, maps, zc);
        else if (cpt == 2) k_diffuse_fs_tma<Real, 2, false><<<grid, blk, b2, st>>>(a, maps, zc);
        else if (sumfs) k_diffuse_fs_tma<Real, 1, true><<<grid, blk, b1, st>>>(a, maps, zc);
        else k_diffuse_fs_tma<Real, 1, false><<<grid, blk, b1, st>>>(a, maps, zc);
    } else {
        k_diffuse_fs<Real, false><<<grid, dim3(DTX, DTY), 0, st>>>(a, zc);
    }
}

// Tiles of the TMA stencil launch, each of which leaves its sum of the new
// fraction solid in a.d.fs_part; 0 when the step runs another variant.
long long stencil_parts(const KernelArgs &a, const TmaHolder &tma)
{
    if (!tma.ok || a.d.rec_flags || !a.d.fs_part) return 0;
    const Geo &g = a.g;
    const int tile_x = DTX * (tma.cpt == 2 ? 2 : 1);
    int zc = tma.zc > 0 ? (tma.zc < g.gz ? tma.zc : g.gz) : pick_zchunk(g, tile_x);
    if (zc > 64) zc = 64;
    return (long long)((g.gx + tile_x - 1) / tile_x) * ((g.gy + DTY - 1) / DTY) * ((g.gz + zc - 1) / zc);
}

long long stencil_parts_max(const Geo &g)
{
    return (long long)((g.gx + DTX - 1) / DTX) * ((g.gy + DTY - 1) / DTY) * g.gz;
}

int launch_stencil(const KernelArgs &a, const TmaHolder &tma, int precision, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (precision == MMS_PREC_F32) launch_stencil_t<float>(a, tma, st);
    else launch_stencil_t<double>(a, tma, st);
    return 1;
}

// The kernels of a step before the stencil (nucleation, activation,
// curvature) and after it (list, capture).
template <typename Real>
static int launch_pre_t(const KernelArgs &a, cudaStream_t st, int start_stage, Profiler *prof)
{
    int n = 0;
    const Geo &g = a.g;
    if (start_stage == 0 && a.d.nsites > 0) {
        // nucleation, and activation in the block that finishes last
        PROF_BEGIN(KID_NUC);
        k_nuc_act<Real><<<a.d.nuc_blocks, NUC_NT, 0, st>>>(a);
        PROF_END(KID_NUC);
        n++;
    } else {
        PROF_BEGIN(KID_ACT);
        k_act<<<1, ACT_NT, 0, st>>>(a, a.d.act_scratch);
        PROF_END(KID_ACT);
        n++;
    }
    if (a.p.tip_curv) {
        long long tot = (long long)g.nranks * g.sbcells;
        PROF_BEGIN(KID_CURV);
        k_curv<Real><<<(int)((tot + 255) / 256), 256, 0, st>>>(a);
        PROF_END(KID_CURV);
        n++;
    }
    return n;
}

template <typename Real>
static int launch_post_t(const KernelArgs &a, cudaStream_t st, Profiler *prof)
{
    const Geo &g = a.g;
    int nblocks = (int)(g.blocks_per_rank * g.nranks);
    PROF_BEGIN(KID_LIST);
    k_list<<<nblocks, LIST_NT, 0, st>>>(a, nblocks);
    PROF_END(KID_LIST);
    PROF_BEGIN(KID_CAPTURE);
    k_capture<Real><<<148 * 8, LIST_NT, 0, st>>>(a);
    PROF_END(KID_CAPTURE);
    return 2;
}

template <typename Real>
static int launch_step_t(const KernelArgs &a, const TmaHolder &tma, cudaStream_t st, int start_stage, Profiler *prof,
                         bool sumfs)
{
    int n = launch_pre_t<Real>(a, st, start_stage, prof);
    PROF_BEGIN(KID_DIFFUSE_FS);
    launch_stencil_t<Real>(a, tma, st, sumfs);
    PROF_END(KID_DIFFUSE_FS);
    n++;
    return n + launch_post_t<Real>(a, st, prof);
}

template <typename Real>
static int launch_slab_phase_t(const KernelArgs &a, const TmaHolder &tma, cudaStream_t st, int phase, int resume)
{
    int n = 0;
    if (phase == 0) {
        if (!resume && a.d.nsites > 0) {
            k_nuc<Real><<<a.d.nuc_blocks, NUC_NT, 0, st>>>(a);
            n++;
        }
        k_act_local<<<1, ACT_NT, 0, st>>>(a);
        return n + 1;
    }
    if (phase == 1) {
        k_act_slab<<<1, ACT_NT, 0, st>>>(a);
        launch_stencil_t<Real>(a, tma, st);
        return 2;
    }
    k_slab_merge<<<1, 256, 0, st>>>(a);
    return 1 + launch_post_t<Real>(a, st, nullptr);
}

int launch_slab_phase(const KernelArgs &a, const TmaHolder &tma, int precision, void *stream, int phase, int resume)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (precision == MMS_PREC_F32) return launch_slab_phase_t<float>(a, tma, st, phase, resume);
    return launch_slab_phase_t<double>(a, tma, st, phase, resume);
}

int launch_curv(const KernelArgs &a, int precision, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    const long long tot = (long long)a.g.nranks * a.g.sbcells;
    if (precision == MMS_PREC_F32) k_curv<float><<<(int)((tot + 255) / 256), 256, 0, st>>>(a);
    else k_curv<double><<<(int)((tot + 255) / 256), 256, 0, st>>>(a);
    return 1;
}

int launch_step_pre(const KernelArgs &a, int precision, void *stream, int start_stage)
{
    cudaStream_t st = (cudaStream_t)stream;
    Profiler *prof = nullptr;
    if (precision == MMS_PREC_F32) return launch_pre_t<float>(a, st, start_stage, prof);
    return launch_pre_t<double>(a, st, start_stage, prof);
}

int launch_step_post(const KernelArgs &a, int precision, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    Profiler *prof = nullptr;
    if (precision == MMS_PREC_F32) return launch_post_t<float>(a, st, prof);
    return launch_post_t<double>(a, st, prof);
}

size_t batch_item_bytes() { return sizeof(BatchItem); }

long long fill_batch_item(void *dst, const KernelArgs &a, const TmaHolder &tma, long long tile_begin)
{
    BatchItem it;
    std::memset(&it, 0, sizeof it);
    std::memcpy(&it.maps, tma.bytes, sizeof(TmaMaps));
    it.a = a;
    const Geo &g = a.g;
    const int tile_x = DTX * (tma.cpt == 2 ? 2 : 1);
    int zc = tma.zc > 0 ? (tma.zc < g.gz ? tma.zc : g.gz) : pick_zchunk(g, tile_x);
    if (zc > 64) zc = 64;
    it.tiles_x = (g.gx + tile_x - 1) / tile_x;
    it.tiles_y = (g.gy + DTY - 1) / DTY;
    it.zchunk = zc;
    it.tile_begin = tile_begin;
    std::memcpy(dst, &it, sizeof it);
    return (long long)it.tiles_x * it.tiles_y * ((g.gz + zc - 1) / zc);
}

template <typename Real, int CPT>
static int batch_grid_t()
{
    constexpr int bytes = Depth<Real, CPT>::TS * Stage<Real, CPT>::BYTES;
    cudaFuncSetAttribute(k_diffuse_fs_batch<Real, CPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_diffuse_fs_batch<Real, CPT>, DTX * DTY, bytes);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (per_sm > 0 ? per_sm : 1) * sms;
}

int batch_grid(int precision, int cpt)
{
    if (precision == MMS_PREC_F32) return cpt == 2 ? batch_grid_t<float, 2>() : batch_grid_t<float, 1>();
    return cpt == 2 ? batch_grid_t<double, 2>() : batch_grid_t<double, 1>();
}

// Blocks per domain of the batched small kernels (0 for a domain that
// launches no such kernel).
int batch_blocks(const KernelArgs &a, int which)
{
    const Geo &g = a.g;
    switch (which) {
    case 0: return a.d.nsites > 0 ? a.d.nuc_blocks : 0;                       // k_nuc
    case 1: return 1;                                                          // k_act
    case 2: return (int)(g.blocks_per_rank * g.nranks);                       // k_list
    default: {                                                                 // k_capture
        long long nb = ((long long)g.gx * g.gy * g.gz) / (LIST_NT * 64);
        return (int)(nb < 1 ? 1 : (nb > 148 * 8 ? 148 * 8 : nb));
    }
    }
}

size_t batch_item_args_offset() { return offsetof(BatchItem, a); }

int launch_small_batch(int which, const void *items, const int *begin, int n, int total, int precision,
                       void *stream)
{
    if (total <= 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    const void *args = (const unsigned char *)items + offsetof(BatchItem, a);
    const size_t stride = sizeof(BatchItem);
    switch (which) {
    case 0:
        if (precision == MMS_PREC_F32) k_nuc_batch<float><<<total, NUC_NT, 0, st>>>(args, stride, begin, n);
        else k_nuc_batch<double><<<total, NUC_NT, 0, st>>>(args, stride, begin, n);
        break;
    case 1: k_act_batch<<<total, ACT_NT, 0, st>>>(args, stride, begin, n); break;
    case 2: k_list_batch<<<total, LIST_NT, 0, st>>>(args, stride, begin, n); break;
    default:
        if (precision == MMS_PREC_F32) k_capture_batch<float><<<total, LIST_NT, 0, st>>>(args, stride, begin, n);
        else k_capture_batch<double><<<total, LIST_NT, 0, st>>>(args, stride, begin, n);
    }
    return 1;
}

int launch_stencil_batch(const void *items, int nitems, long long total_tiles, int precision, int cpt, int grid,
                         void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    const BatchItem *it = (const BatchItem *)items;
    if (precision == MMS_PREC_F32) {
        if (cpt == 2)
            k_diffuse_fs_batch<float, 2><<<grid, dim3(DTX, DTY), Depth<float, 2>::TS * Stage<float, 2>::BYTES, st>>>(
                it, nitems, total_tiles);
        else
            k_diffuse_fs_batch<float, 1><<<grid, dim3(DTX, DTY), Depth<float, 1>::TS * Stage<float, 1>::BYTES, st>>>(
                it, nitems, total_tiles);
    } else {
        if (cpt == 2)
            k_diffuse_fs_batch<double, 2><<<grid, dim3(DTX, DTY), Depth<double, 2>::TS * Stage<double, 2>::BYTES,
                                            st>>>(it, nitems, total_tiles);
        else
            k_diffuse_fs_batch<double, 1><<<grid, dim3(DTX, DTY), Depth<double, 1>::TS * Stage<double, 1>::BYTES,
                                            st>>>(it, nitems, total_tiles);
    }
    return 1;
}

int launch_step(const KernelArgs &a, const TmaHolder &tma, int precision, void *stream, int start_stage, Profiler *prof,
                bool sumfs)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (precision == MMS_PREC_F32) return launch_step_t<float>(a, tma, st, start_stage, prof, sumfs);
    return launch_step_t<double>(a, tma, st, start_stage, prof, sumfs);
}

int launch_temp_am(const KernelArgs &a, const AmParams &m, int precision, void *stream, Profiler *prof, int rows)
{
    cudaStream_t st = (cudaStream_t)stream;
    const Geo &g = a.g;
    const long long tab = (long long)AM_NT * (g.gx + g.gy + g.gz + 6);
    auto grid_of = [&](int tx, int tr) {
        return dim3((unsigned)((g.gx + 2 + tx - 1) / tx), (unsigned)(((long long)(g.gy + 2) * (g.gz + 2) + tr - 1) / tr));
    };
    int n = 1;
    PROF_BEGIN(KID_TEMP_AM);
    if (precision == MMS_PREC_F32) {
        // tables in FP32; the contraction on the tensor cores (am_tc.cu)
        k_am_tables<float><<<(unsigned)((tab + 255) / 256), 256, 0, st>>>(a, m);
        n += launch_am_contract_tc(a, m, st, rows);
    } else {
        using T = AmTile<double>;
        k_am_tables<double><<<(unsigned)((tab + 255) / 256), 256, 0, st>>>(a, m);
        k_am_contract<double><<<grid_of(T::XL * T::MX, AMC_NT / T::XL * T::MY), AMC_NT, 0, st>>>(a, m);
        n++;
    }
    PROF_END(KID_TEMP_AM);
    return n;
}

// Folds the per-block (sum, compensation) pairs in a fixed order.
// Thread 0 gets the total of nb (sum, compensation) pairs, folded in a
// fixed order (strided per thread, then lanes, then the 32 warps, each
// merge a TwoSum); every thread of the 1024 must call it.
__device__ __forceinline__ double fold_pairs(const double *partial, int nb)
{
    __shared__ double ws[32], wc[32];
    double s = 0, c = 0;
    for (int b = threadIdx.x; b < nb; b += 1024) {
        const double x = partial[2 * b];
        const double t = s + x, bp = t - s;
        c += (s - (t - bp)) + (x - bp) + partial[2 * b + 1];
        s = t;
    }
    auto merge = [&](double x, double xc) {
        const double t = s + x, bp = t - s;
        c += xc + ((s - (t - bp)) + (x - bp));
        s = t;
    };
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double x = __shfl_down_sync(FULL_MASK, s, o), xc = __shfl_down_sync(FULL_MASK, c, o);
        merge(x, xc);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        ws[w] = s;
        wc[w] = c;
    }
    __syncthreads();
    if (w == 0) {
        s = ws[lane];
        c = wc[lane];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double x = __shfl_down_sync(FULL_MASK, s, o), xc = __shfl_down_sync(FULL_MASK, c, o);
            merge(x, xc);
        }
    }
    return s + c;
}

__global__ void __launch_bounds__(1024) k_reduce_fold(double *partial, int nb)
{
    const double v = fold_pairs(partial, nb);
    if (threadIdx.x == 0) partial[2 * nb] = v;
}

// The same fold, written with the step's control block straight into
// host memory the device can address (no copies after the kernel).
__global__ void __launch_bounds__(1024) k_fold_out(const double *partial, int nb, const Ctl *ctl, double *host_sum,
                                                   Ctl *host_ctl)
{
    const double v = fold_pairs(partial, nb);
    static_assert(sizeof(Ctl) % sizeof(unsigned long long) == 0, "Ctl is copied in 8-byte words");
    constexpr int W = (int)(sizeof(Ctl) / sizeof(unsigned long long));
    if (threadIdx.x < W)
        ((unsigned long long *)host_ctl)[threadIdx.x] = ((const volatile unsigned long long *)ctl)[threadIdx.x];
    if (threadIdx.x == 0) *host_sum = v;
}

// Folds the last step's per-tile fraction-solid sums (stencil_parts of
// them) and copies the total to pinned memory; the caller synchronises.
int launch_fold_fs(const KernelArgs &a, long long nparts, void *stream, double *pinned)
{
    cudaStream_t st = (cudaStream_t)stream;
    k_reduce_fold<<<1, 1024, 0, st>>>(a.d.fs_part, (int)nparts);
    cudaMemcpyAsync(pinned, a.d.fs_part + 2 * nparts, sizeof(double), cudaMemcpyDeviceToHost, st);
    return 1;
}

int launch_fold_fs_out(const KernelArgs &a, long long nparts, void *stream, double *host_sum, void *host_ctl)
{
    k_fold_out<<<1, 1024, 0, (cudaStream_t)stream>>>(a.d.fs_part, (int)nparts, a.d.ctl, host_sum, (Ctl *)host_ctl);
    return 1;
}

// Blocks of k_reduce that are resident at once (at most RED_BLOCKS): every
// warp then takes the same number of rows, give or take one.
template <typename Real>
static int reduce_grid()
{
    // computed once, thread-safely (a static initialised by a call)
    static const int nb = [] {
        int per_sm = 0, dev = 0, sms = 148;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_reduce<Real>, RED_NT, 0);
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int v = (per_sm > 0 ? per_sm : 1) * sms;
        return v < RED_BLOCKS ? v : RED_BLOCKS;
    }();
    return nb;
}

int launch_reduce(const KernelArgs &a, int precision, int what, double *host_out, void *stream, double *pinned)
{
    cudaStream_t st = (cudaStream_t)stream;
    const int nb = precision == MMS_PREC_F32 ? reduce_grid<float>() : reduce_grid<double>();
    double *partial = a.d.red;
    if (precision == MMS_PREC_F32) k_reduce<float><<<nb, RED_NT, 0, st>>>(a, what, partial);
    else k_reduce<double><<<nb, RED_NT, 0, st>>>(a, what, partial);
    k_reduce_fold<<<1, 1024, 0, st>>>(partial, nb);
    cudaMemcpyAsync(pinned, partial + 2 * nb, sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    *host_out = *pinned;
    if (precision == MMS_PREC_F32 && what == MMS_REDUCE_CE_SUM)  // deviations from Cinit were summed
        *host_out += a.p.cinit * (double)((long long)a.g.gx * a.g.gy * a.g.gz);
    return 2;
}

// Rows of row_bytes bytes from one pitch to another (the reference's halo'd
// layout to the padded device layout and back), 4-byte words when possible.
__global__ void k_repack(unsigned char *__restrict__ dst, long long dst_pitch, const unsigned char *__restrict__ src,
                         long long src_pitch, int row_bytes, long long rows)
{
    for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
        unsigned char *d = dst + r * dst_pitch;
        const unsigned char *q = src + r * src_pitch;
        if ((row_bytes & 3) == 0 && (dst_pitch & 3) == 0 && (src_pitch & 3) == 0) {
            for (int w = threadIdx.x; w < row_bytes / 4; w += blockDim.x) ((unsigned *)d)[w] = ((const unsigned *)q)[w];
        } else {
            for (int b = threadIdx.x; b < row_bytes; b += blockDim.x) d[b] = q[b];
        }
    }
}

int launch_repack(void *dst, long long dst_pitch, const void *src, long long src_pitch, int row_bytes, long long rows,
                  void *stream)
{
    const long long nb = rows < 148 * 64 ? rows : 148 * 64;
    k_repack<<<(unsigned)(nb > 0 ? nb : 1), 256, 0, (cudaStream_t)stream>>>(
        (unsigned char *)dst, dst_pitch, (const unsigned char *)src, src_pitch, row_bytes, rows);
    return 1;
}

int launch_compute_d(const KernelArgs &a, int precision, double *dev_out, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    int nb = (int)((a.g.N + 255) / 256);
    if (precision == MMS_PREC_F32) k_compute_d<float><<<nb, 256, 0, st>>>(a, dev_out);
    else k_compute_d<double><<<nb, 256, 0, st>>>(a, dev_out);
    return 1;
}

int launch_fill_temperature(const KernelArgs &a, double *dev_out, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    int nb = (int)((a.g.N + 255) / 256);
    k_fill_temperature<<<nb, 256, 0, st>>>(a, dev_out);
    return 1;
}

int launch_convert_ref(const KernelArgs &a, int precision, int field, int to_device, double *ref_f64, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    const long long rows = (long long)(a.g.gy + 2) * (a.g.gz + 2);
    const int nb = (int)(rows < 148LL * 16 ? rows : 148LL * 16);
    if (precision == MMS_PREC_F32) k_convert_ref<float><<<nb, 256, 0, st>>>(a, field, to_device, ref_f64);
    else k_convert_ref<double><<<nb, 256, 0, st>>>(a, field, to_device, ref_f64);
    return 1;
}

int launch_convert(const KernelArgs &a, int precision, int field, int to_device, double *dev_f64,
                   void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    int nb = (int)((a.g.N + 255) / 256);
    if (precision == MMS_PREC_F32) k_convert<float><<<nb, 256, 0, st>>>(a, field, to_device, dev_f64);
    else k_convert<double><<<nb, 256, 0, st>>>(a, field, to_device, dev_f64);
    return 1;
}

}  // namespace mms
