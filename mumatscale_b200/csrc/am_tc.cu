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

// bounded (about a second)
__device__ __forceinline__ bool tc_bar_wait(unsigned long long *bar, unsigned parity)
{
    for (unsigned it = 0; it < (1u << 22); it++) {
        if (tc_bar_try(bar, parity)) return true;
        if (it > 32) __nanosleep(256);
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

// tile width: the fewest tiles of at most 256 x cells, rounded up to 32
// (the epilogue splits a tile's columns in two halves of 16-column loads)
int am_tc_tile_n(int nx)
{
    const int ntx = (nx + TC_NMAX - 1) / TC_NMAX;
    int n = (nx + ntx - 1) / ntx;
    return (n + 31) / 32 * 32;
}

// the kernel's shared-memory size; called once per context at set-up (not
// during stream capture)
int am_tc_prepare()
{
    return cudaFuncSetAttribute(k_am_contract_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM) ==
           cudaSuccess;
}

int launch_am_contract_tc(const KernelArgs &a, const AmParams &m, void *stream)
{
    const Geo &g = a.g;
    const int nx = g.gx + 2;
    const int N = am_tc_tile_n(nx);
    dim3 grid((unsigned)((nx + N - 1) / N), (unsigned)(((long long)(g.gy + 2) * (g.gz + 2) + TC_M - 1) / TC_M));
    k_am_contract_tc<<<grid, TC_NT, TC_SMEM, (cudaStream_t)stream>>>(a, m, N);
    return 1;
}

}  // namespace mms
