// am_tc.cu — the AM temperature contraction of the FP32 form on the
// 5th-generation tensor cores.
//
//   T[row, x] = liniT + Tfront sum_i YZ[row, i] X[i, x],   YZ = Y_i(y) Z_i(z)
//
// is a (rows x 400) by (400 x nx) matrix product.  A CTA computes a tile of
// 128 rows by N x cells (N <= 256, a multiple of 32) with tcgen05.mma
// kind::tf32, accumulating in tensor memory.  TF32 keeps 10 mantissa bits,
// so every operand is split as v = hi + lo (hi = v rounded to TF32, lo the
// exact FP32 remainder) and the product is hi*hi + hi*lo + lo*hi, three MMAs
// per step of 8 nodes; the dropped lo*lo term and lo's own TF32 rounding are
// ~2^-22 relative.
//
// Per chunk of 16 nodes the threads write the split operands into one of two
// shared-memory buffers in the K-major, no-swizzle layout of the tensor core
// (8 x 16-byte core matrices: rows 16 B apart, the two 16-byte halves of a
// row's 8 nodes 128 B apart, 8-row groups 256 B apart), fence them to the
// async proxy, and one thread issues the MMAs and commits them to the
// buffer's mbarrier; a buffer is written again only after that barrier
// (waited on with a bound) shows its MMAs complete, so the staging of one
// chunk overlaps the MMAs of the previous one.
// The epilogue reads the accumulators with tcgen05.ld (warp w sees TMEM lanes
// 32 (w mod 4) ...) and writes T.
#include <cuda.h>
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "mms_internal.h"

namespace mms {

constexpr int TC_M = 128;          // rows per tile (MMA M)
constexpr int TC_NMAX = 256;       // x cells per tile at most (MMA N)
constexpr int TC_KC = 16;          // nodes per shared-memory chunk
constexpr int TC_KS = TC_KC / 8;   // MMA K-steps per chunk
constexpr int TC_NT = 256;
constexpr int TC_A_BYTES = TC_M * 8 * 4;       // one K-step of A (one part)
constexpr int TC_B_BYTES = TC_NMAX * 8 * 4;    // one K-step of B (one part), room for N = 256
constexpr int TC_SET = 2 * TC_KS * TC_A_BYTES + 2 * TC_KS * TC_B_BYTES;  // hi and lo of A and B
constexpr int TC_SMEM = 2 * TC_SET;            // two chunks in flight

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// v rounded to TF32 (10 mantissa bits, ties away from zero) and the remainder
__device__ __forceinline__ void tf32_split(float v, float &hi, float &lo)
{
    const unsigned u = (__float_as_uint(v) + 0x1000u) & 0xffffe000u;
    hi = __uint_as_float(u);
    lo = v - hi;
}

// byte offset of element (r, k) (k < 8) in a K-major no-swizzle operand block
__device__ __forceinline__ int kmajor_off(int r, int k)
{
    return (r >> 3) * 256 + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4;
}

// shared-memory matrix descriptor: start >> 4, leading-dimension byte offset
// 128 (the second 16-byte half of the K-step), stride byte offset 256 (the
// next 8-row group), descriptor version 1, no swizzle
__device__ __forceinline__ unsigned long long kmajor_desc(unsigned saddr)
{
    return (unsigned long long)((saddr >> 4) & 0x3fffu) | ((unsigned long long)(128 >> 4) << 16) |
           ((unsigned long long)(256 >> 4) << 32) | (1ULL << 46);
}

__device__ __forceinline__ void tc_mma(unsigned dtmem, unsigned long long adesc, unsigned long long bdesc,
                                       unsigned idesc, unsigned accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(dtmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tc_commit(unsigned long long *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool tc_bar_try(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded (2^22 polls, about a second); try_wait suspends the thread in
// hardware between polls, so only a long wait backs off with short sleeps
__device__ __forceinline__ bool tc_bar_wait(unsigned long long *bar, unsigned parity)
{
    for (unsigned it = 0; it < (1u << 22); it++) {
        if (tc_bar_try(bar, parity)) return true;
        if (it > (1u << 14)) __nanosleep(64);
    }
    return false;
}

__global__ void __launch_bounds__(TC_NT, 2) k_am_contract_tc(KernelArgs a, AmParams m, int N)
{
    const Ctl *ctl = a.d.ctl;
    if (stalled(ctl)) return;
    extern __shared__ __align__(1024) unsigned char tsm[];
    __shared__ __align__(8) unsigned long long bar[2];
    __shared__ unsigned tmem_base;
    __shared__ int s_abort;
    const Geo &g = a.g;
    const Phys &p = a.p;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nx = g.gx + 2, ny = g.gy + 2, nz = g.gz + 2;
    const float *__restrict__ X = (const float *)a.d.am_tab;
    const float *__restrict__ Y = X + (long long)AM_NT * nx;
    const float *__restrict__ Z = Y + (long long)AM_NT * ny;
    const int *zon = (const int *)(Z + (long long)AM_NT * nz);
    const int x0 = blockIdx.x * N;
    const long long r0 = (long long)blockIdx.y * TC_M;
    const long long nrows = (long long)ny * nz;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_base)),
                     "r"(256u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned dtmem = tmem_base;
    // kind::tf32, F32 accumulate, A and B K-major, M = 128, N
    const unsigned idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(N >> 3) << 17) | ((unsigned)(TC_M >> 4) << 24);

    // staging: A (YZ products) by row srow, nodes sk0, sk0 + 2, ...; B (X) by
    // column tid for tid < N, every node of the chunk
    const int srow = tid & (TC_M - 1), sk0 = tid >> 7;
    const long long row = r0 + srow;
    const bool rin = row < nrows;
    const int Kr = rin ? (int)(row / ny) : 0, Jr = rin ? (int)(row - (long long)Kr * ny) : 0;
    const float *Yr = Y + Jr, *Zr = Z + Kr;
    const bool bcol = tid < N && x0 + tid < nx;
    const float *Xc = X + (x0 + (tid < N ? tid : 0));

    unsigned ph[2] = {0u, 0u};
    int step = 0, c = 0;
    // operands of the next chunk, loaded one chunk ahead so that their
    // latency overlaps the stores, fences and MMA issue of the current one
    float av[TC_KC / 2], bv[TC_KC];
    auto load_chunk = [&](int i0) {
#pragma unroll
        for (int j = 0; j < TC_KC / 2; j++) {
            const int k = sk0 + 2 * j;
            av[j] = rin ? __ldg(Yr + (long long)(i0 + k) * ny) * __ldg(Zr + (long long)(i0 + k) * nz) : 0.f;
        }
#pragma unroll
        for (int k = 0; k < TC_KC; k++) bv[k] = bcol ? __ldg(Xc + (long long)(i0 + k) * nx) : 0.f;
    };
    load_chunk(0);
    for (int i0 = 0; i0 < AM_NT; i0 += TC_KC, c++) {
        const int b = c & 1;
        unsigned char *set = tsm + b * TC_SET;
        unsigned char *A_hi = set, *A_lo = set + TC_KS * TC_A_BYTES;
        unsigned char *B_hi = set + 2 * TC_KS * TC_A_BYTES, *B_lo = B_hi + TC_KS * TC_B_BYTES;
        // this buffer's previous MMAs (chunk c - 2) must be complete
        if (c >= 2) {
            if (!tc_bar_wait(&bar[b], ph[b])) s_abort = 1;
            ph[b] ^= 1u;
        }
        __syncthreads();
        if (s_abort) break;
#pragma unroll
        for (int j = 0; j < TC_KC / 2; j++) {
            const int k = sk0 + 2 * j;
            float hi, lo;
            tf32_split(av[j], hi, lo);
            const int off = (k >> 3) * TC_A_BYTES + kmajor_off(srow, k & 7);
            *(float *)(A_hi + off) = hi;
            *(float *)(A_lo + off) = lo;
        }
        if (tid < N) {
#pragma unroll
            for (int k = 0; k < TC_KC; k++) {
                float hi, lo;
                tf32_split(bv[k], hi, lo);
                const int off = (k >> 3) * TC_B_BYTES + kmajor_off(tid, k & 7);
                *(float *)(B_hi + off) = hi;
                *(float *)(B_lo + off) = lo;
            }
        }
        if (i0 + TC_KC < AM_NT) load_chunk(i0 + TC_KC);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (int s2 = 0; s2 < TC_KS; s2++) {
                const unsigned long long ah = kmajor_desc(smem_addr(A_hi + s2 * TC_A_BYTES));
                const unsigned long long al = kmajor_desc(smem_addr(A_lo + s2 * TC_A_BYTES));
                const unsigned long long bh = kmajor_desc(smem_addr(B_hi + s2 * TC_B_BYTES));
                const unsigned long long bl = kmajor_desc(smem_addr(B_lo + s2 * TC_B_BYTES));
                tc_mma(dtmem, ah, bh, idesc, step > 0 ? 1u : 0u);
                tc_mma(dtmem, ah, bl, idesc, 1u);
                tc_mma(dtmem, al, bh, idesc, 1u);
                step++;
            }
            tc_commit(&bar[b]);
        }
    }
    // the last chunk of each buffer (bounded waits; after an abort these
    // drain whatever is still in flight before the tensor memory is freed)
    for (int b = 0; b < 2 && b < c; b++) {
        const int last = (c - 1 - b);       // chunks c-1 and c-2
        const int bb = last & 1;
        if (!tc_bar_wait(&bar[bb], ph[bb])) s_abort = 1;
        ph[bb] ^= 1u;
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (s_abort) {
        if (tid == 0) raise_error(a.d.ctl, MMS_ERR_TIMEOUT);
    } else {
        // epilogue: warp w reads TMEM lanes 32 (w mod 4) .. + 31 (its rows),
        // columns of its half of the tile, 16 at a time
        const AmStep st = am_step(p, m, ctl->timestep + 1);
        const int q = warp & 3, half = warp >> 2;
        const int rowl = 32 * q + lane;
        const long long rrow = r0 + rowl;
        const bool ok = rrow < nrows;
        const int K = ok ? (int)(rrow / ny) : 0, J = ok ? (int)(rrow - (long long)K * ny) : 0;
        const bool on = ok && zon[K] != 0;
        const int c0 = half * (N / 2), c1 = (half + 1) * (N / 2);
        for (int cc = c0; cc < c1; cc += 16) {
            unsigned v[16];
            const unsigned taddr = dtmem + ((unsigned)(32 * q) << 16) + (unsigned)cc;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (ok) {
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const int x = x0 + cc + j;
                    if (cc + j >= c1 || x >= nx) break;
                    const long long cell = (long long)K * g.sz + (long long)J * g.sy + x;
                    const double T = on ? st.liniT + st.Tfront * (double)__uint_as_float(v[j]) : 0.0;
                    a.d.T[cell] = T;
                    if (a.d.lsindex && T > p.Tliq) a.d.lsindex[cell] = 1;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(dtmem), "r"(256u) : "memory");
    }
}

// ----------------------------------------------------------------------------
// Persistent, warp-specialised form.  The product is computed transposed,
//
//   T^T[x, row] = sum_i X[i, x] YZ[row, i],
//
// so the operand shared by every CTA (X, one 400 x gx table per step) is the
// MMA's A side (M = 128 x cells) and is written once per step, already split
// into TF32 head and remainder and laid out as the tensor core reads it, by
// k_am_tables (am_ximg); a CTA brings a chunk of it in with one
// cp.async.bulk.  The B side, N (<= 256) (y, z) rows of YZ products, is
// formed by four producer warps straight into shared memory.  A tile is 128
// x cells by N rows; its accumulator takes N of the 512 tensor-memory
// columns, so the epilogue of one tile (four more warps: tcgen05.ld, then T
// and the layer flag) runs while the next tile accumulates in the other
// half.  Warp 0 loads A, warp 1 issues the MMAs (one thread), warps 2-5
// produce B, warps 6-9 drain the accumulators.  Per stage (16 nodes): A 16
// KB, B 32 KB; four stages in flight.  The halo columns x = 0 and gx + 1
// (outside the 128-cell x tiles) are summed on the CUDA cores by the
// epilogue warps while their first accumulator fills.
//
// Every wait is bounded; on expiry a thread raises MMS_ERR_TIMEOUT and sets a
// shared abort flag that ends every other role's waits, then each role
// drains what it has in flight (bulk copies, committed MMAs) before the
// tensor memory is freed.
constexpr int T2_M = 128;                       // x cells per tile (MMA M)
constexpr int T2_NMAX = 256;                    // (y, z) rows per tile (MMA N) at most
constexpr int T2_KC = 16;                       // nodes per stage
constexpr int T2_KS = T2_KC / 8;                // MMA K-steps per stage
constexpr int T2_S = 4;                         // stages
constexpr int T2_NCH = AM_NT / T2_KC;           // stages per tile
constexpr int T2_A_KS = T2_M * 8 * 4;           // one K-step, one part (head or remainder) of A
constexpr int T2_B_KS = T2_NMAX * 8 * 4;        // the same of B (room for N = 256)
constexpr int T2_A = T2_KS * 2 * T2_A_KS;       // A bytes per stage
constexpr int T2_STAGE = T2_A + T2_KS * 2 * T2_B_KS;
constexpr int T2_SMEM = T2_S * T2_STAGE + 128;  // + alignment of the ring
constexpr int T2_NT = 320;
constexpr int T2_PROD0 = 64, T2_EPI0 = 192;     // first thread of the producers / epilogue
static_assert(AM_NT % T2_KC == 0, "nodes per stage");

// the A image of one step: [x tile][K-step (50)][head, remainder][128 x 8]
__host__ __device__ constexpr long long am_ximg_floats(int gx)
{
    return (long long)((gx + T2_M - 1) / T2_M) * (AM_NT / 8) * 2 * (T2_M * 8);
}

__device__ __forceinline__ void t2_arrive(unsigned long long *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void t2_arrive_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void t2_bulk_load(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Bounded wait (about a second) that also gives up as soon as another role
// has raised the abort flag; `strict` waits ignore the flag (draining).
__device__ __forceinline__ bool t2_wait(unsigned long long *bar, unsigned parity, volatile int *abort,
                                        bool strict = false)
{
    for (unsigned it = 0; it < (1u << 22); it++) {
        if (tc_bar_try(bar, parity)) return true;
        if (!strict && (it & 31) == 31 && *abort) return false;
        if (it > (1u << 14)) __nanosleep(64);
    }
    *abort = 1;
    return false;
}

struct T2Tile {
    int xt;          // x tile: cells 1 + 128 xt ...
    long long r0;    // first (y, z) row
};

__device__ __forceinline__ T2Tile t2_tile(long long t, int ntx, int N)
{
    T2Tile w;
    w.xt = (int)(t % ntx);
    w.r0 = (t / ntx) * (long long)N;
    return w;
}

__global__ void __launch_bounds__(T2_NT, 1)
    k_am_contract_tc2(const __grid_constant__ KernelArgs a, const __grid_constant__ AmParams m, int N, int ntx,
                      long long ntiles)
{
    Ctl *ctl = a.d.ctl;
    if (stalled(ctl)) return;
    extern __shared__ unsigned char t2_raw[];
    unsigned char *ring = (unsigned char *)(((unsigned long long)t2_raw + 127) & ~127ULL);
    __shared__ __align__(8) unsigned long long fullA[T2_S], fullB[T2_S], empty[T2_S], accf[2], acce[2];
    __shared__ unsigned tmem_base;
    __shared__ int s_abort;
    const Geo &g = a.g;
    const Phys &p = a.p;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nx = g.gx + 2, ny = g.gy + 2, nz = g.gz + 2;
    const float *__restrict__ X = (const float *)a.d.am_tab;
    const float *__restrict__ Y = X + (long long)AM_NT * nx;
    const float *__restrict__ Z = Y + (long long)AM_NT * ny;
    const int *zon = (const int *)(Z + (long long)AM_NT * nz);
    const float *__restrict__ ximg = a.d.am_ximg;
    const long long nrows = (long long)ny * nz;
    volatile int *abort = &s_abort;

    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_base)),
                     "r"(512u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s2 = 0; s2 < T2_S; s2++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&fullA[s2])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;" ::"r"(smem_addr(&fullB[s2])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&empty[s2])) : "memory");
        }
        for (int b = 0; b < 2; b++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&accf[b])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;" ::"r"(smem_addr(&acce[b])) : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = tmem_base;

    if (warp == 0) {
        // ---- A: one bulk copy of 16 KB per stage
        if (lane == 0) {
            long long q = 0;
            bool ok = true;
            for (long long t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                const T2Tile w = t2_tile(t, ntx, N);
                const float *src = ximg + (long long)w.xt * (AM_NT / 8) * 2 * (T2_M * 8);
                for (int c = 0; c < T2_NCH; c++, q++) {
                    const int s2 = (int)(q % T2_S);
                    if (q >= T2_S && !t2_wait(&empty[s2], (unsigned)((q / T2_S - 1) & 1), abort)) {
                        ok = false;
                        break;
                    }
                    t2_arrive_tx(&fullA[s2], (unsigned)T2_A);
                    t2_bulk_load(ring + s2 * T2_STAGE, src + (long long)c * T2_KS * 2 * (T2_M * 8), (unsigned)T2_A,
                                 &fullA[s2]);
                }
            }
            // copies still in flight land before the CTA may exit
            for (long long j = (q > T2_S ? q - T2_S : 0); j < q; j++)
                t2_wait(&fullA[j % T2_S], (unsigned)((j / T2_S) & 1), abort, true);
        }
    } else if (warp == 1) {
        // ---- MMA issue (one thread)
        if (lane == 0) {
            // kind::tf32, F32 accumulate, A and B K-major, M = 128, N
            const unsigned idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(N >> 3) << 17) |
                                   ((unsigned)(T2_M >> 4) << 24);
            long long q = 0, tl = 0;
            unsigned long long *last = nullptr;
            unsigned last_par = 0;
            bool ok = true;
            for (long long t = blockIdx.x; t < ntiles && ok; t += gridDim.x, tl++) {
                const int b = (int)(tl & 1);
                if (tl >= 2 && !t2_wait(&acce[b], (unsigned)((tl / 2 - 1) & 1), abort)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const unsigned d = tmem + (unsigned)(b * T2_NMAX);
                for (int c = 0; c < T2_NCH; c++, q++) {
                    const int s2 = (int)(q % T2_S);
                    const unsigned par = (unsigned)((q / T2_S) & 1);
                    if (!t2_wait(&fullA[s2], par, abort) || !t2_wait(&fullB[s2], par, abort)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    unsigned char *A = ring + s2 * T2_STAGE, *B = A + T2_A;
#pragma unroll
                    for (int k = 0; k < T2_KS; k++) {
                        const unsigned long long ah = kmajor_desc(smem_addr(A + (2 * k) * T2_A_KS));
                        const unsigned long long al = kmajor_desc(smem_addr(A + (2 * k + 1) * T2_A_KS));
                        const unsigned long long bh = kmajor_desc(smem_addr(B + (2 * k) * T2_B_KS));
                        const unsigned long long bl = kmajor_desc(smem_addr(B + (2 * k + 1) * T2_B_KS));
                        tc_mma(d, ah, bh, idesc, (c > 0 || k > 0) ? 1u : 0u);
                        tc_mma(d, ah, bl, idesc, 1u);
                        tc_mma(d, al, bh, idesc, 1u);
                    }
                    tc_commit(&empty[s2]);
                    last = &empty[s2];
                    last_par = par;
                }
                if (!ok) break;
                tc_commit(&accf[b]);
                last = &accf[b];
                last_par = (unsigned)((tl / 2) & 1);
            }
            // every committed MMA completes before the tensor memory is freed
            if (last) t2_wait(last, last_par, abort, true);
        }
    } else if (tid < T2_EPI0) {
        // ---- B: (y, z) rows pr and pr + 128 of the tile, 16 nodes per stage
        const int pr = tid - T2_PROD0;
        long long q = 0;
        bool ok = true;
        for (long long t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
            const T2Tile w = t2_tile(t, ntx, N);
            int J[2], K[2];
            bool on[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int n = pr + 128 * h;
                const long long R = w.r0 + n;
                on[h] = n < N && R < nrows;
                K[h] = on[h] ? (int)(R / ny) : 0;
                J[h] = on[h] ? (int)(R - (long long)K[h] * ny) : 0;
            }
            for (int c = 0; c < T2_NCH; c++, q++) {
                const int s2 = (int)(q % T2_S);
                float v[2][T2_KC];
#pragma unroll
                for (int h = 0; h < 2; h++)
#pragma unroll
                    for (int k = 0; k < T2_KC; k++) {
                        const int i = c * T2_KC + k;
                        v[h][k] = on[h] ? __ldg(Y + (long long)i * ny + J[h]) * __ldg(Z + (long long)i * nz + K[h])
                                        : 0.f;
                    }
                if (q >= T2_S && !t2_wait(&empty[s2], (unsigned)((q / T2_S - 1) & 1), abort)) {
                    ok = false;
                    break;
                }
                unsigned char *B = ring + s2 * T2_STAGE + T2_A;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int n = pr + 128 * h;
                    if (n >= N) continue;
                    const int off = (n >> 3) * 256 + (n & 7) * 16;
#pragma unroll
                    for (int k = 0; k < T2_KS; k++) {
                        float hi[8], lo[8];
#pragma unroll
                        for (int e = 0; e < 8; e++) tf32_split(v[h][8 * k + e], hi[e], lo[e]);
                        unsigned char *bh = B + (2 * k) * T2_B_KS + off, *bl = B + (2 * k + 1) * T2_B_KS + off;
                        *(float4 *)bh = make_float4(hi[0], hi[1], hi[2], hi[3]);
                        *(float4 *)(bh + 128) = make_float4(hi[4], hi[5], hi[6], hi[7]);
                        *(float4 *)bl = make_float4(lo[0], lo[1], lo[2], lo[3]);
                        *(float4 *)(bl + 128) = make_float4(lo[4], lo[5], lo[6], lo[7]);
                    }
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                t2_arrive(&fullB[s2]);
            }
        }
    } else {
        // ---- epilogue: warp w reads tensor-memory lanes 32 (w mod 4) .. + 31
        const int qd = warp & 3, e = tid - T2_EPI0;
        const int xl = 32 * qd + lane;
        const AmStep st = am_step(p, m, ctl->timestep + 1);
        long long tl = 0;
        for (long long t = blockIdx.x; t < ntiles; t += gridDim.x, tl++) {
            const T2Tile w = t2_tile(t, ntx, N);
            const int b = (int)(tl & 1);
            // halo columns of the rows of this tile, while the accumulator fills
            for (int hx = 0; hx < 2; hx++) {
                const int xh = hx == 0 ? 0 : nx - 1;
                if ((hx == 0 && w.xt != 0) || (hx == 1 && w.xt != ntx - 1)) continue;
                for (int n = e; n < N; n += 128) {
                    const long long R = w.r0 + n;
                    if (R >= nrows) break;
                    const int K = (int)(R / ny), J = (int)(R - (long long)K * ny);
                    float acc = 0.f;
                    if (zon[K])
                        for (int i = 0; i < AM_NT; i++)
                            acc = fmaf(__ldg(X + (long long)i * nx + xh),
                                       __ldg(Y + (long long)i * ny + J) * __ldg(Z + (long long)i * nz + K), acc);
                    const long long cell = (long long)K * g.sz + (long long)J * g.sy + xh;
                    const double T = zon[K] ? st.liniT + st.Tfront * (double)acc : 0.0;
                    a.d.T[cell] = T;
                    if (a.d.lsindex && T > p.Tliq) a.d.lsindex[cell] = 1;
                }
            }
            const bool got = t2_wait(&accf[b], (unsigned)((tl / 2) & 1), abort);
            // the warp-wide tcgen05.ld below needs the whole warp, converged
            if (!__all_sync(0xffffffffu, got)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int x = 1 + T2_M * w.xt + xl;
            const bool xin = x <= g.gx;
            long long R = w.r0;
            int K = (int)(R / ny), J = (int)(R - (long long)K * ny);
            for (int cc = 0; cc < N; cc += 16) {
                unsigned v[16];
                const unsigned taddr = tmem + ((unsigned)(32 * qd) << 16) + (unsigned)(b * T2_NMAX + cc);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                    "%12, %13, %14, %15}, [%16];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                      "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                      "=r"(v[14]), "=r"(v[15])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    if (xin && R < nrows) {
                        const long long cell = (long long)K * g.sz + (long long)J * g.sy + x;
                        const bool on = zon[K] != 0;
                        const double T = on ? st.liniT + st.Tfront * (double)__uint_as_float(v[j]) : 0.0;
                        a.d.T[cell] = T;
                        if (a.d.lsindex && T > p.Tliq) a.d.lsindex[cell] = 1;
                    }
                    R++;
                    if (++J == ny) {
                        J = 0;
                        K++;
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            t2_arrive(&acce[b]);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (s_abort && tid == 0) raise_error(ctl, MMS_ERR_TIMEOUT);
    if (warp == 1) {
        __syncwarp();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
    }
}

// Rows per tile: the multiple of 16 (128 .. 256) whose tiles, dealt to one
// persistent CTA per SM, leave the fewest rows on the busiest CTA.
static int t2_rows_per_tile(long long nrows, int ntx, int nsm)
{
    int best = T2_NMAX;
    long long best_load = -1;
    for (int n = T2_NMAX; n >= 128; n -= 16) {
        const long long tiles = ntx * ((nrows + n - 1) / n);
        const long long load = ((tiles + nsm - 1) / nsm) * n;
        if (best_load < 0 || load < best_load) {
            best_load = load;
            best = n;
        }
    }
    return best;
}

static int sm_count()
{
    static int n = [] {
        int dev = 0, v = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
            v = 148;
        return v;
    }();
    return n;
}

// tile width: the fewest tiles of at most 256 x cells, rounded up to 32
// (the epilogue splits a tile's columns in two halves of 16-column loads)
int am_tc_tile_n(int nx)
{
    const int ntx = (nx + TC_NMAX - 1) / TC_NMAX;
    int n = (nx + ntx - 1) / ntx;
    return (n + 31) / 32 * 32;
}

// the kernels' shared-memory sizes; called once per context at set-up (not
// during stream capture)
int am_tc_prepare()
{
    sm_count();
    return cudaFuncSetAttribute(k_am_contract_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM) ==
               cudaSuccess &&
           cudaFuncSetAttribute(k_am_contract_tc2, cudaFuncAttributeMaxDynamicSharedMemorySize, T2_SMEM) ==
               cudaSuccess;
}

long long am_ximg_size(int gx) { return am_ximg_floats(gx); }

int launch_am_contract_tc(const KernelArgs &a, const AmParams &m, void *stream)
{
    const Geo &g = a.g;
    if (a.d.am_ximg) {
        const int ntx = (g.gx + T2_M - 1) / T2_M;
        const long long nrows = (long long)(g.gy + 2) * (g.gz + 2);
        const int nsm = sm_count();
        const int N = t2_rows_per_tile(nrows, ntx, nsm);
        const long long ntiles = (long long)ntx * ((nrows + N - 1) / N);
        const unsigned grid = (unsigned)(ntiles < nsm ? ntiles : nsm);
        k_am_contract_tc2<<<grid, T2_NT, T2_SMEM, (cudaStream_t)stream>>>(a, m, N, ntx, ntiles);
        return 1;
    }
    const int nx = g.gx + 2;
    const int N = am_tc_tile_n(nx);
    dim3 grid((unsigned)((nx + N - 1) / N), (unsigned)(((long long)(g.gy + 2) * (g.gz + 2) + TC_M - 1) / TC_M));
    k_am_contract_tc<<<grid, TC_NT, TC_SMEM, (cudaStream_t)stream>>>(a, m, N);
    return 1;
}

}  // namespace mms
