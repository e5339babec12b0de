// am_tc.cu — the AM temperature contraction of the FP32 form on the
// 5th-generation tensor cores.
//
//   T[x, row] = liniT + Tfront sum_i X_i(x) YZ_i(row),   YZ_i(row) = Y_i(y) Z_i(z)
//
// over the 400 quadrature nodes i of the moving-source model
// (temperature.c:62-123) is a (x cells x 400) by (400 x rows) matrix product.
// A CTA computes tiles of 128 x cells (MMA M, the A side) by N (y, z) rows
// (MMA N, the B side) with tcgen05.mma kind::f16 on FP16 operands,
// accumulating in FP32 in tensor memory.
//
// Operands.  FP16 keeps 11 significant bits, so every operand is split as
// v = hi + lo (hi = v rounded to FP16, lo the FP16 rounding of the
// remainder) and the product is hi*hi + hi*lo + lo*hi, three MMAs per step
// of 16 nodes; the dropped lo*lo term and lo's rounding are ~2^-22 relative.
// The operands are scaled into FP16's range by powers of two (exact): X <= 1
// by 2^14, and Y Z by am_b_scale, which maps its upper bound ldt / Tl_0 to at
// most 2^14; FP16's subnormals keep an absolute resolution of 2^-24, 2^-38 of
// the scaled maximum, so one scale per operand serves every row and column.
// The epilogue divides the scales out.  Against the TF32 x 3 form this
// halves the MMAs (K = 16 per instruction instead of 8) and the operand
// bytes moved through shared memory.
//
// Accumulation.  The tensor core adds an MMA's products and the accumulator
// with truncation, so each MMA into an accumulator loses up to one unit in
// the last place of the running sum, always toward zero.  Two measures keep
// that small: the hi*hi products go to one accumulator and the ~2^-11
// smaller cross products to another (so the large sum takes 25 MMAs, not
// 75), and the nodes are summed from the oldest (widest, smallest terms) to
// the most recent, so that a cell's largest terms are added last, onto a sum
// that is still small.  The epilogue adds the two accumulators and forms
// liniT + Tfront sum in FP32 with the constants split into head and
// remainder (within one unit in the last place of the FP32 result).
//
// Operand images.  Both operands reach shared memory by bulk copies of
// images written once per step, already scaled, split into FP16 head and
// remainder and laid out as the tensor core reads them: k_am_tables writes
// the X image (x blocks of 128), k_am_bimg the B image (blocks of N (y, z)
// rows, 1.6 KB per row).  The B image is the larger (53 MB at 512 x 256 x
// 128) but is written at memory bandwidth by a plain elementwise kernel and
// read by the contraction from L2 (the x blocks of a row block are
// consecutive tiles); forming it inside the contraction took four warps per
// SM whose serial per-stage work set the pace.
//
// Persistent, warp-specialised, one CTA per SM:
//   warp 0       both operands: per stage one bulk copy from each image
//   warp 1       the MMAs (one thread), committed to mbarriers
//   warps 2-9    epilogue: tcgen05.ld of both accumulators, T (kept in FP32
//                in this form) and the layer flag to global memory; two
//                warps per group of 32 tensor-memory lanes, each taking every
//                other 16 columns
// Stages of two K-steps (32 nodes; the last stage of a tile holds the one
// K-step left of 25) circulate in a shared-memory ring: seven of 32 KB with
// N = 128, four of 48 KB with N = 256.  A stage costs each role a fixed
// handshake (a barrier wait, index arithmetic, a commit or an arrival) of
// several hundred cycles, so the stages are as large as the ring allows.  With N = 128 the 512
// tensor-memory columns hold two sets of accumulators, so a tile's epilogue
// runs while the next tile accumulates; with N = 256 one set fills them.
//
// The halo columns x = 0 and gx + 1 are not computed here: no kernel of a
// step reads the temperature there.  k_am_halo fills them from the same
// tables where they are read (the temperature download, and every step when
// the multi-layer flag lsindex is kept).
//
// Every wait is bounded; on expiry a thread raises MMS_ERR_TIMEOUT and sets
// a shared abort flag that ends every other role's waits, then each role
// drains what it has in flight (bulk copies, committed MMAs) before the
// tensor memory is freed.
#include <cstring>

#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "mms_internal.h"

namespace mms {

constexpr int TC_M = 128;                  // x cells per tile (MMA M)
constexpr int TC_KE = 16;                  // nodes per MMA K-step (FP16 operands)
constexpr int TC_NKS = AM_NT / TC_KE;      // K-steps per tile
constexpr int TC_A_KS = TC_M * TC_KE * 2;  // one K-step, one part (head or remainder) of A, bytes
constexpr int TC_A_CH = 2 * TC_A_KS;       // one K-step of A, both parts: a chunk of the operand image
constexpr int TC_NT = 320;
constexpr int TC_EPI0 = 64;                  // first thread of the epilogue
constexpr int TC_NEPI = TC_NT - TC_EPI0;     // epilogue threads (eight warps)
static_assert(AM_NT % TC_KE == 0, "nodes per K-step");

template <int NB>
struct TcCfg {
    static constexpr int KS = 2;                            // K-steps per stage
    static constexpr int NCH = (TC_NKS + KS - 1) / KS;      // stages per tile (the last may hold fewer)
    static constexpr int B_KS = NB * TC_KE * 2;             // one K-step, one part of B, bytes, at N = NB
    static constexpr int A_ST = KS * TC_A_CH;               // A bytes of a full stage
    static constexpr int STAGE = A_ST + KS * 2 * B_KS;      // 32 KB (N = 128) or 48 KB (N = 256)
    static constexpr int S = NB == 128 ? 7 : 4;             // stages in the ring
    // 256-row tiles: the epilogue hands T to the tensor-store engine through
    // staging buffers (two per group of four warps, 16 rows x 128 x cells
    // of FP32 each), so that its stores drain while the next tile's MMAs run
    static constexpr bool TST = NB == 256;
    static constexpr int STG_BYTES = 16 * TC_M * 4;
    static constexpr int STG = TST ? 4 * STG_BYTES : 0;
    static constexpr int SMEM = S * STAGE + STG + 128;      // + alignment of the ring
    static constexpr int BUFS = NB == 128 ? 2 : 1;          // accumulator sets (2 NB columns each)
    // Stage c holds the K-steps (16-node chunks of the node order) lo(c) ..
    // lo(c) + nk(c) - 1: the stages run from the oldest nodes (the highest
    // chunks) to the most recent, and the last one holds what is left.
    static __device__ __forceinline__ int lo(int c)
    {
        const int l = TC_NKS - KS * (c + 1);
        return l > 0 ? l : 0;
    }
    static __device__ __forceinline__ int nk(int c) { return TC_NKS - KS * c - lo(c); }
};

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor of a K-major, no-swizzle operand block (8 x
// 16-byte core matrices: rows 16 B apart, the two 16-byte halves of a row's 8
// nodes 128 B apart, 8-row groups 256 B apart): start >> 4, leading-dimension
// byte offset 128, stride byte offset 256, descriptor version 1
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
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
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

__device__ __forceinline__ void tc_arrive(unsigned long long *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void tc_arrive_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void tc_bulk_load(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Bounded wait (2^22 polls, about a second) that also gives up as soon as
// another role has raised the abort flag; `strict` waits ignore the flag
// (draining).  try_wait suspends the thread in hardware between polls, so
// only a long wait backs off with short sleeps.
__device__ __forceinline__ bool tc_wait(unsigned long long *bar, unsigned parity, volatile int *abort,
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

// v as a head of 11 significant bits and the FP16 rounding of the
// remainder, packed by two.  The head is Veltkamp's split (t = (2^13 + 1) v,
// head = t - (t - v), with every operation rounded on its own): v = head +
// remainder exactly in FP32, and the head converts to FP16 exactly wherever
// FP16 holds 11 bits (|head| >= 2^-14; below that the conversion's error is
// at most 2^-25, FP16's subnormal resolution).  Two conversions per pair
// instead of four (no conversion of the head back to FP32): the conversion
// pipe is the narrow one here.
__device__ __forceinline__ void half_split2(float v0, float v1, unsigned &hi, unsigned &lo)
{
    const float t0 = __fmul_rn(v0, 8193.f), t1 = __fmul_rn(v1, 8193.f);
    const float h0 = __fsub_rn(t0, __fsub_rn(t0, v0)), h1 = __fsub_rn(t1, __fsub_rn(t1, v1));
    const __half2 h = __floats2half2_rn(h0, h1);
    const __half2 l = __floats2half2_rn(__fsub_rn(v0, h0), __fsub_rn(v1, h1));
    hi = *(const unsigned *)&h;
    lo = *(const unsigned *)&l;
}

static_assert(TC_M == 128, "am_ximg_part lays the X image out in 128-cell tiles");

// 16 consecutive tensor-memory columns of this warp's 32 lanes
__device__ __forceinline__ void tmem_ld16(unsigned taddr, unsigned (&v)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}

// Waits for this thread's tcgen05.ld in flight; the registers they fill are
// operands, so that no use of them is scheduled before the wait.
__device__ __forceinline__ void tmem_wait_ld(unsigned (&a)[16], unsigned (&b)[16])
{
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]),
                   "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]),
                   "+r"(a[15]), "+r"(b[0]), "+r"(b[1]), "+r"(b[2]), "+r"(b[3]), "+r"(b[4]), "+r"(b[5]), "+r"(b[6]),
                   "+r"(b[7]), "+r"(b[8]), "+r"(b[9]), "+r"(b[10]), "+r"(b[11]), "+r"(b[12]), "+r"(b[13]),
                   "+r"(b[14]), "+r"(b[15])
                 :
                 : "memory");
}

template <int NB>
__global__ void __launch_bounds__(TC_NT, 1)
    k_am_contract_tc(const __grid_constant__ KernelArgs a, const __grid_constant__ AmParams m, int N, int ntx,
                     long long ntiles, const __grid_constant__ CUtensorMap tmap, int tst)
{
    using C = TcCfg<NB>;
    constexpr int S = C::S;
    Ctl *ctl = a.d.ctl;
    if (stalled(ctl)) return;
    extern __shared__ unsigned char tc_raw[];
    unsigned char *ring = (unsigned char *)(((unsigned long long)tc_raw + 127) & ~127ULL);
    // full[s]: the stage's A and B copies have landed (one arrival with
    // their byte count); empty[s]: the MMAs that read the stage are done
    __shared__ __align__(8) unsigned long long full[S], empty[S], accf[2], acce[2];
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
    const long long nrows = (long long)ny * nz;
    volatile int *abort = &s_abort;

    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_base)),
                     "r"(512u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < S; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&full[s])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&empty[s])) : "memory");
        }
        for (int b = 0; b < 2; b++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&accf[b])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&acce[b])), "r"(TC_NEPI)
                         : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = tmem_base;

    // The roles count stages with a ring slot s and the parity ph of its
    // current round: full[s] completes once per round (wait on ph); a slot is
    // refilled once empty[s] has completed the previous round (wait on ph ^ 1).
    // B's bytes per K-step and part at this tile height
    const int BN = N * TC_KE * 2;
    if (warp == 0) {
        // ---- A and B: per stage one bulk copy of its K-steps' chunks from
        // each operand image (contiguous in node order): X's image for the
        // tile's x block, the B image for its row block
        if (lane == 0) {
            unsigned s = 0, ph = 0, issued = 0;
            bool ok = true;
            const unsigned char *bimg = am_bimg(a.d.am_ximg, g.gx, g.gy, g.gz);
            for (long long t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                const int xt = (int)(t % ntx);
                const long long rb = t / ntx;
                const unsigned char *srcA = (const unsigned char *)a.d.am_ximg + (long long)xt * TC_NKS * TC_A_CH;
                const unsigned char *srcB = bimg + rb * TC_NKS * 2 * BN;
                for (int c = 0; c < C::NCH; c++) {
                    if (issued >= (unsigned)S && !tc_wait(&empty[s], ph ^ 1u, abort)) {
                        ok = false;
                        break;
                    }
                    const unsigned ba = (unsigned)(C::nk(c) * TC_A_CH), bb = (unsigned)(C::nk(c) * 2 * BN);
                    tc_arrive_tx(&full[s], ba + bb);
                    tc_bulk_load(ring + s * C::STAGE, srcA + C::lo(c) * TC_A_CH, ba, &full[s]);
                    tc_bulk_load(ring + s * C::STAGE + C::A_ST, srcB + C::lo(c) * 2 * BN, bb, &full[s]);
                    issued++;
                    if (++s == (unsigned)S) s = 0, ph ^= 1u;
                }
            }
            // copies still in flight land before the CTA may exit
            for (unsigned j = (issued > (unsigned)S ? issued - S : 0); j < issued; j++)
                tc_wait(&full[j % S], (j / S) & 1u, abort, true);
        }
    } else if (warp == 1) {
        // ---- MMA issue (one thread)
        if (lane == 0) {
            // kind::f16 with FP16 A and B, F32 accumulate, both K-major, M = 128, N
            // (idesc2: N = 2 N, B's head and remainder as one operand: in the
            // stage the remainder's rows follow the head's)
            const unsigned idesc = (1u << 4) | (0u << 7) | (0u << 10) | ((unsigned)(N >> 3) << 17) |
                                   ((unsigned)(TC_M >> 4) << 24);
            const bool pair_b = 2 * N <= 256;
            const unsigned idesc2 = (1u << 4) | (0u << 7) | (0u << 10) | ((unsigned)((2 * N) >> 3) << 17) |
                                    ((unsigned)(TC_M >> 4) << 24);
            // descriptors of the ring's operands: the start address field is
            // the byte address / 16 (below 2^14 for any shared address), so a
            // stage's descriptors are the ring's plus the offset / 16
            const unsigned long long d0 = kmajor_desc(smem_addr(ring));
            unsigned s = 0, ph = 0, tl = 0;
            unsigned long long *last = nullptr;
            unsigned last_par = 0;
            bool ok = true;
            for (long long t = blockIdx.x; t < ntiles && ok; t += gridDim.x, tl++) {
                const int b = C::BUFS == 2 ? (int)(tl & 1) : 0;
                const unsigned use = C::BUFS == 2 ? tl >> 1 : tl;  // earlier tiles in this set
                if (use >= 1 && !tc_wait(&acce[b], (use - 1) & 1u, abort)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const unsigned dhh = tmem + (unsigned)(b * 2 * NB), dxx = dhh + (unsigned)N;
                for (int c = 0; c < C::NCH; c++) {
                    if (!tc_wait(&full[s], ph, abort)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const unsigned long long da = d0 + (unsigned)((s * C::STAGE) >> 4);
                    const unsigned long long db = da + (unsigned)(C::A_ST >> 4);
                    const int n = C::nk(c);
#pragma unroll
                    for (int kk = 0; kk < C::KS; kk++) {
                        if (kk >= n) break;
                        const int k = n - 1 - kk;  // the later (older) K-step of the stage first
                        const unsigned long long ah = da + (unsigned)((2 * k) * TC_A_KS >> 4);
                        const unsigned long long al = da + (unsigned)((2 * k + 1) * TC_A_KS >> 4);
                        const unsigned long long bh = db + (unsigned)((2 * k) * BN >> 4);
                        const unsigned long long bl = db + (unsigned)((2 * k + 1) * BN >> 4);
                        const unsigned acc = (c > 0 || kk > 0) ? 1u : 0u;
                        if (pair_b) {
                            // the head and remainder of B are rows 0..N-1 and
                            // N..2N-1 of one 2N-row operand, and the cross
                            // accumulator is the hh one's next N columns: one
                            // MMA gives hi*hi and hi*lo, a second adds lo*hi
                            tc_mma(dhh, ah, bh, idesc2, acc);
                            tc_mma(dxx, al, bh, idesc, 1u);
                        } else {
                            tc_mma(dhh, ah, bh, idesc, acc);
                            tc_mma(dxx, ah, bl, idesc, acc);
                            tc_mma(dxx, al, bh, idesc, 1u);
                        }
                    }
                    tc_commit(&empty[s]);
                    last = &empty[s];
                    last_par = ph;
                    if (++s == (unsigned)S) s = 0, ph ^= 1u;
                }
                if (!ok) break;
                tc_commit(&accf[b]);
                last = &accf[b];
                last_par = use & 1u;
            }
            // every committed MMA completes before the tensor memory is freed
            if (last) tc_wait(last, last_par, abort, true);
        }
    } else {
        // ---- epilogue: warp w reads tensor-memory lanes 32 (w mod 4) .. + 31
        // (its 32 x cells); of each tile's 16-column chunks (rows), warps
        // 2-5 take the even ones and warps 6-9 the odd ones, loading the next
        // chunk while the current one is stored
        const int qd = warp & 3, hf = (warp - TC_EPI0 / 32) >> 2;
        const int xl = 32 * qd + lane;
        const AmStep st = am_step(p, m, ctl->timestep + 1);
        // the sums are of (2^14 X) (sB YZ): back to X YZ, times Tfront.  T =
        // liniT + tf sum in FP32 with tf and liniT each as a head and the
        // FP32 rounding of its remainder: two roundings (the FMA of the heads
        // and the final addition) against one for the FP64 form of the same
        // expression, no FP32-FP64 conversions
        const double tf = st.Tfront / (16384.0 * am_b_scale(st));
        const float tf_h = (float)tf, tf_l = (float)(tf - (double)tf_h);
        const float li_h = (float)st.liniT, li_l = (float)(st.liniT - (double)li_h);
        // kernel parameters in registers: a store through T32 might alias
        // the parameter block as far as the compiler knows, so every read of
        // it after a store would be a load again
        float *const T32 = a.d.T32;
        int *const lsx = a.d.lsindex;
        const double Tliq = p.Tliq;
        const long long sy = g.sy, sz = g.sz;
        const int gx = g.gx;
        // tensor stores: this group's staging buffers, the chunks it has
        // staged (the same count in its four warps), its issuing thread
        const bool use_tst = C::TST && tst && !lsx;
        float *const stg = (float *)(ring + S * C::STAGE + hf * 2 * C::STG_BYTES);
        unsigned staged = 0;
        const bool issuer = qd == 0 && lane == 0;
        const unsigned bar_id = 1 + hf;
        long long tl = 0;
        for (long long t = blockIdx.x; t < ntiles; t += gridDim.x, tl++) {
            const int xt = (int)(t % ntx);
            const long long r0 = (t / ntx) * (long long)N;
            const int b = C::BUFS == 2 ? (int)(tl & 1) : 0;
            const long long use = C::BUFS == 2 ? tl / 2 : tl;
            // the tile's first row and the flags of its z plane and the next
            // (the rows cross at most one plane when ny >= N), read before
            // the wait so that the loads are not on the chunks' path
            const int K0 = (int)(r0 / ny), J0 = (int)(r0 - (long long)K0 * ny);
            const bool on0 = zon[K0] != 0, on1 = K0 + 1 < nz && zon[K0 + 1] != 0;
            // the warp-wide tcgen05.ld below needs the whole warp, converged;
            // with tensor stores the four warps of a group (which meet at
            // named barriers) leave together too
            bool got = __all_sync(0xffffffffu, tc_wait(&accf[b], (unsigned)(use & 1), abort));
            if (C::TST) {
                unsigned all;
                asm volatile(
                    "{\n\t.reg .pred p, q;\n\t"
                    "setp.ne.u32 q, %1, 0;\n\t"
                    "bar.red.and.pred p, %2, 128, q;\n\t"
                    "selp.u32 %0, 1, 0, p;\n\t}"
                    : "=r"(all)
                    : "r"(got ? 1u : 0u), "r"(bar_id)
                    : "memory");
                got = all != 0;
            }
            if (!got) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int x = 1 + TC_M * xt + xl;
            const bool xin = x <= gx;
            const unsigned col = tmem + ((unsigned)(32 * qd) << 16) + (unsigned)(b * 2 * NB);
            // T of rows r0 + cc .. + 15 from the chunk's two accumulators.  The
            // sixteen values are formed first, free of the row walk's
            // branches, so that their arithmetic overlaps; then they are
            // stored, in one run when the rows stay in one z plane.
            auto store16 = [&](int cc, const unsigned (&vh)[16], const unsigned (&vx)[16]) {
                int Jc = J0 + cc, Kc = K0;
                bool onc = on0;
                if (Jc >= ny) Jc -= ny, Kc++, onc = on1;
                if (use_tst && ny >= N && Jc + 16 <= ny) {
                    // the chunk's 16 rows lie in plane Kc (rows past the last
                    // plane and x cells past gx are outside the tensor map and
                    // not written): stage them, then one thread of the group
                    // issues the tensor store
                    float *buf = stg + (staged & 1) * (C::STG_BYTES / 4);
#pragma unroll
                    for (int j = 0; j < 16; j++) {
                        const float sum = __uint_as_float(vh[j]) + __uint_as_float(vx[j]);
                        const float T = __fadd_rn(__fmaf_rn(tf_h, sum, li_h), __fmaf_rn(tf_l, sum, li_l));
                        buf[j * TC_M + xl] = onc ? T : 0.f;
                    }
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    asm volatile("bar.sync %0, 128;" ::"r"(bar_id) : "memory");
                    if (issuer) {
                        asm volatile(
                            "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
                                (unsigned long long)&tmap),
                            "r"(4 + TC_M * xt), "r"(Jc), "r"(Kc), "r"(smem_addr(buf))
                            : "memory");
                        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                        // the buffer the next chunk fills was read by the store before this one
                        asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
                    }
                    asm volatile("bar.sync %0, 128;" ::"r"(bar_id) : "memory");
                    staged++;
                    return;
                }
                if (!xin) return;
                float Tv[16];
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    // the two accumulators (the cross sum is ~2^-11 of the other)
                    const float sum = __uint_as_float(vh[j]) + __uint_as_float(vx[j]);
                    Tv[j] = __fadd_rn(__fmaf_rn(tf_h, sum, li_h), __fmaf_rn(tf_l, sum, li_l));
                }
                long long R = r0 + cc;
                if (ny >= N && R + 16 <= nrows) {
                    int J = J0 + cc, K = K0;
                    bool on = on0;
                    if (J >= ny) J -= ny, K++, on = on1;
                    if (J + 16 <= ny) {
                        float *const out = T32 + ((long long)K * sz + (long long)J * sy + x);
#pragma unroll
                        for (int j = 0; j < 16; j++) {
                            const float T = on ? Tv[j] : 0.f;
                            out[j * sy] = T;
                            if (lsx && (double)T > Tliq) lsx[(out - T32) + j * sy] = 1;
                        }
                        return;
                    }
                }
                int K = (int)(R / ny), J = (int)(R - (long long)K * ny);
                long long cell = (long long)K * sz + (long long)J * sy + x;
                bool on = zon[K] != 0;
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    if (R < nrows) {
                        const float T = on ? Tv[j] : 0.f;
                        T32[cell] = T;
                        if (lsx && (double)T > Tliq) lsx[cell] = 1;
                    }
                    R++;
                    cell += sy;
                    if (++J == ny) {
                        J = 0;
                        K++;
                        cell += sz - (long long)ny * sy;
                        on = K < nz && zon[K] != 0;
                    }
                }
            };
            // the accumulator set is released as soon as this thread's last
            // tensor-memory load has completed, before that chunk is stored
            bool released = false;
            auto release = [&]() {
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                tc_arrive(&acce[b]);
                released = true;
            };
            unsigned ha[16], xa[16], hb[16], xb[16];
            int cc = 16 * hf;
            if (cc < N) {
                tmem_ld16(col + (unsigned)cc, ha);
                tmem_ld16(col + (unsigned)(N + cc), xa);
            }
            tmem_wait_ld(ha, xa);
            while (cc < N) {
                const int c1 = cc + 32;
                if (c1 < N) {
                    tmem_ld16(col + (unsigned)c1, hb);
                    tmem_ld16(col + (unsigned)(N + c1), xb);
                } else {
                    release();
                }
                store16(cc, ha, xa);
                if (c1 >= N) break;
                tmem_wait_ld(hb, xb);
                const int c2 = c1 + 32;
                if (c2 < N) {
                    tmem_ld16(col + (unsigned)c2, ha);
                    tmem_ld16(col + (unsigned)(N + c2), xa);
                } else {
                    release();
                }
                store16(c1, hb, xb);
                if (c2 >= N) break;
                tmem_wait_ld(ha, xa);
                cc = c2;
            }
            if (!released) release();
        }
        // the tensor stores complete (their shared-memory reads and their
        // writes) before the CTA leaves
        if (C::TST && issuer) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
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

// The B operand image of a step: for every (y, z) row R (row R mod N of
// block R / N) and K-step k, the 16 scaled products sB Y_i(y) Z_i(z) of the
// K-step's nodes as FP16 head and remainder, in the layout the contraction's
// stages copy as they are (the rows of the last block past the last row are
// zero).  Grid: x over rows (consecutive rows across a warp), y over
// K-steps.  The Y and Z rows come from the node-contiguous copies
// k_am_tables writes, the scale from the word it leaves after its step
// marker.
__global__ void __launch_bounds__(256) k_am_bimg(const __grid_constant__ KernelArgs a,
                                                 const __grid_constant__ AmParams m, int N)
{
    const Ctl *ctl = a.d.ctl;
    if (stalled(ctl)) return;
    const Geo &g = a.g;
    const int nx = g.gx + 2, ny = g.gy + 2, nz = g.gz + 2;
    // the step's scale, which k_am_tables leaves after its step marker
    const float *tabs = (const float *)a.d.am_tab;
    const int *zon = (const int *)(tabs + (long long)AM_NT * (nx + ny + nz));
    (void)m;
    const unsigned nrows = (unsigned)ny * (unsigned)nz, rp = (nrows + N - 1) / N * N;
    const unsigned R = blockIdx.x * blockDim.x + threadIdx.x;
    if (R >= rp) return;
    const int k = blockIdx.y;
    const unsigned rb = R / (unsigned)N;
    const int n = (int)(R - rb * (unsigned)N), BN = N * TC_KE * 2;
    uint4 h0 = make_uint4(0, 0, 0, 0), h1 = h0, l0 = h0, l1 = h0;
    if (R < nrows) {
        const unsigned K = R / (unsigned)ny, J = R - K * (unsigned)ny;
        const float4 *y = (const float4 *)(am_yt(a.d.am_ximg, g.gx) + (long long)J * AM_NT + k * TC_KE);
        const float4 *z = (const float4 *)(am_zt(a.d.am_ximg, g.gx, g.gy) + (long long)K * AM_NT + k * TC_KE);
        const float sB = *am_tab_sb(zon, nz);
        unsigned hi[8], lo[8];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const float4 yv = __ldg(y + q), zv = __ldg(z + q);
            half_split2(yv.x * zv.x * sB, yv.y * zv.y * sB, hi[2 * q], lo[2 * q]);
            half_split2(yv.z * zv.z * sB, yv.w * zv.w * sB, hi[2 * q + 1], lo[2 * q + 1]);
        }
        h0 = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        h1 = make_uint4(hi[4], hi[5], hi[6], hi[7]);
        l0 = make_uint4(lo[0], lo[1], lo[2], lo[3]);
        l1 = make_uint4(lo[4], lo[5], lo[6], lo[7]);
    }
    unsigned char *dst = am_bimg(a.d.am_ximg, g.gx, g.gy, g.gz) + ((long long)rb * TC_NKS + k) * 2 * BN +
                         (n >> 3) * 256 + (n & 7) * 16;
    *(uint4 *)dst = h0;
    *(uint4 *)(dst + 128) = h1;
    *(uint4 *)(dst + BN) = l0;
    *(uint4 *)(dst + BN + 128) = l1;
}

// Temperature of the halo columns x = 0 and gx + 1 from the tables of step
// ctl->timestep + ahead (FP32 form): the sum over the nodes in node order
// with fused multiply-adds, into out (a temperature download buffer) or,
// when out is null, into the FP32 temperature field with the layer flag.
// One thread per (column, row); rows are consecutive across a warp, so the Y
// loads coalesce.  Nothing is written when the tables were built for
// another step.
__global__ void __launch_bounds__(256) k_am_halo(KernelArgs a, AmParams m, double *out, int ahead)
{
    const Ctl *ctl = a.d.ctl;
    const Geo &g = a.g;
    const Phys &p = a.p;
    const int nx = g.gx + 2, ny = g.gy + 2, nz = g.gz + 2;
    const float *__restrict__ X = (const float *)a.d.am_tab;
    const float *__restrict__ Y = X + (long long)AM_NT * nx;
    const float *__restrict__ Z = Y + (long long)AM_NT * ny;
    const int *zon = (const int *)(Z + (long long)AM_NT * nz);
    const unsigned long long ts = ctl->timestep + (unsigned long long)ahead;
    if (*am_tab_step(zon, nz) != ts) return;
    const long long nrows = (long long)ny * nz;
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= 2 * nrows) return;
    const int side = (int)(e / nrows);
    const long long R = e - side * nrows;
    const int K = (int)(R / ny), J = (int)(R - (long long)K * ny);
    const int xh = side == 0 ? 0 : nx - 1;
    float acc = 0.f;
    if (zon[K])
        for (int i = 0; i < AM_NT; i++)
            acc = fmaf(__ldg(X + (long long)i * nx + xh), __ldg(Y + (long long)i * ny + J) * __ldg(Z + (long long)i * nz + K),
                       acc);
    const AmStep st = am_step(p, m, ts);
    const long long cell = (long long)K * g.sz + (long long)J * g.sy + xh;
    const double T = zon[K] ? st.liniT + st.Tfront * (double)acc : 0.0;
    if (out) {
        out[cell] = T;
    } else {
        const float T32 = (float)T;
        a.d.T32[cell] = T32;
        if (a.d.lsindex && (double)T32 > p.Tliq) a.d.lsindex[cell] = 1;
    }
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

// the kernels' shared-memory sizes; called once per context at set-up (not
// during stream capture)
int am_tc_prepare()
{
    sm_count();
    return cudaFuncSetAttribute(k_am_contract_tc<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                TcCfg<128>::SMEM) == cudaSuccess &&
           cudaFuncSetAttribute(k_am_contract_tc<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                TcCfg<256>::SMEM) == cudaSuccess;
}

long long am_ximg_size(int gx, int gy, int gz)
{
    return am_ximg_part(gx) + (long long)(gy + gz + 4) * AM_NT + am_bimg_part(gy, gz);
}

// rows: 256-row tiles (one accumulator set), 64-128 rows (two), 0 = 256
// when the grid has at least two 256-row tiles per SM, else 128.
// With two sets a tile's epilogue overlaps the next tile's MMAs; 256-row
// tiles take fewer, larger MMAs per node (three N = 256 against two N = 256
// and two N = 128 for the same products) and fewer stages, which outweighs
// their epilogue running alone at 512 x 256 x 128 (tables and B image
// included: 128 rows 0.125 ms, 112 0.132, 96 0.139, 80 0.157, 64 0.178, 256
// 0.113); mms_autotune times 128 and 256 on the domain.
int launch_am_contract_tc(const KernelArgs &a, const AmParams &m, void *stream, int rows)
{
    const Geo &g = a.g;
    const int ntx = (g.gx + TC_M - 1) / TC_M;
    const long long nrows = (long long)(g.gy + 2) * (g.gz + 2);
    const int nsm = sm_count();
    if (rows == 0) {
        // 256-row tiles when there are enough of them to keep every SM busy
        // for two, else 128
        const long long wide_tiles = (long long)ntx * ((nrows + 255) / 256);
        rows = wide_tiles >= 2LL * nsm ? 256 : 128;
    }
    const bool wide = rows == 256;
    const int N = wide ? 256 : (rows >= 64 && rows <= 128 ? rows / 16 * 16 : 128);
    const long long ntiles = (long long)ntx * ((nrows + N - 1) / N);
    const unsigned grid = (unsigned)(ntiles < nsm ? ntiles : nsm);
    cudaStream_t st = (cudaStream_t)stream;
    const long long rp = (nrows + N - 1) / N * N;
    k_am_bimg<<<dim3((unsigned)((rp + 255) / 256), TC_NKS), 256, 0, st>>>(a, m, N);
    // the temperature as a tensor-store target for 256-row tiles (the host
    // encodes it at every launch; launches are captured into graphs once)
    CUtensorMap tmap;
    std::memset(&tmap, 0, sizeof tmap);
    const int tst = wide && encode_t32_store(&tmap, a, TC_M, 16) ? 1 : 0;
    if (wide) k_am_contract_tc<256><<<grid, TC_NT, TcCfg<256>::SMEM, st>>>(a, m, N, ntx, ntiles, tmap, tst);
    else k_am_contract_tc<128><<<grid, TC_NT, TcCfg<128>::SMEM, st>>>(a, m, N, ntx, ntiles, tmap, tst);
    int n = 2;
    if (a.d.lsindex) {
        // the layer flag is kept for every cell, halo columns included
        const long long e = 2 * nrows;
        k_am_halo<<<(unsigned)((e + 255) / 256), 256, 0, st>>>(a, m, nullptr, 1);
        n++;
    }
    return n;
}

int launch_am_halo_fill(const KernelArgs &a, const AmParams &m, double *dev_out, void *stream)
{
    const long long e = 2LL * (a.g.gy + 2) * (a.g.gz + 2);
    k_am_halo<<<(unsigned)((e + 255) / 256), 256, 0, (cudaStream_t)stream>>>(a, m, dev_out, 0);
    return 1;
}

}  // namespace mms
