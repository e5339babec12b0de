// adjoint.cu — frozen-CA replay and hand-written adjoint of the continuous
// part of one timestep: diffusion (growth.c:69-162) followed by the fraction-
// solid change (growth.c:220-273), with respect to the solute, liquid
// concentration and fraction-solid fields and to the parameters D_l, k and
// the Gibbs-Thomson coefficient.
//
// Frozen CA.  Everything discrete in a step is taken from a recorded forward
// run: which branch fs_change took in every cell (liquid reset, solid keep,
// growth, growth clamped at fs = 1, growth reset at fs < 0), nucleation and
// capture (which change no continuous value: a captured cell was reset to
// cl = ce, fs = 0 in the same step already), and the curvature used.  With
// those fixed, a step is a smooth map x_t -> x_{t+1} of (ce, cl, fs), and
// its transpose Jacobian is applied here cell by cell.
//
// The replay kernel evaluates the same expressions as the step's stencil
// (kernels.cu, cell_update), in the same order and precision, so with the
// recorded parameters it reproduces the recorded trajectory bit for bit.
#include <cuda.h>
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "mms_internal.h"

namespace mms {

constexpr int ADJ_NT = 256;

__device__ __forceinline__ bool interior_cell(const Geo &g, long long v, int &i, int &j, int &k, long long &c)
{
    long long n = (long long)g.gx * g.gy * g.gz;
    if (v >= n) return false;
    i = (int)(v % g.gx) + 1;
    long long r = v / g.gx;
    j = (int)(r % g.gy) + 1;
    k = (int)(r / g.gy) + 1;
    c = (long long)k * g.sz + (long long)j * g.sy + i;
    return true;
}

// neighbour offsets in the diffusion order +x, -x, +y, -y, +z, -z
__device__ __forceinline__ void nb_offsets(const Geo &g, long long (&o)[6])
{
    o[0] = 1;
    o[1] = -1;
    o[2] = g.sy;
    o[3] = -g.sy;
    o[4] = g.sz;
    o[5] = -g.sz;
}

// Is the n-th neighbour of interior cell (i,j,k) inside the domain?
__device__ __forceinline__ bool nb_inside(const Geo &g, int n, int i, int j, int k)
{
    switch (n) {
    case 0: return i < g.gx;
    case 1: return i > 1;
    case 2: return j < g.gy;
    case 3: return j > 1;
    case 4: return k < g.gz;
    default: return k > 1;
    }
}

// ------------------------------------------------------------------ replay
// x_t (ce0, cl0, fs0) -> x_{t+1} (ce1, cl1, fs1) with the branches of step
// ts (flags) and the curvature it used, under the parameters in p.
template <typename Real>
__global__ void __launch_bounds__(ADJ_NT) k_replay(Geo g, Phys p, const Real *__restrict__ ce0,
                                                   const Real *__restrict__ cl0, const Real *__restrict__ fs0,
                                                   Real *__restrict__ ce1, Real *__restrict__ cl1,
                                                   Real *__restrict__ fs1, const unsigned char *__restrict__ flags,
                                                   const double *__restrict__ curv, unsigned long long ts)
{
    int i, j, k;
    long long c;
    if (!interior_cell(g, blockIdx.x * (long long)ADJ_NT + threadIdx.x, i, j, k, c)) return;
    const PhysR<Real> q = phys_r<Real>(p);
    long long o[6];
    nb_offsets(g, o);
    const Real conc = cl0[c], lspfs = fs0[c], oce = ce0[c];
    Real nb_cl[6], nb_fs[6];
#pragma unroll
    for (int n = 0; n < 6; n++) {
        nb_cl[n] = cl0[c + o[n]];
        nb_fs[n] = fs0[c + o[n]];
    }
    const Real one_x = (Real)(1 - g.padx), one_y = (Real)(1 - g.pady), one_zp = (Real)(1 - g.padz_hi),
               one_zm = (Real)(1 - g.padz_lo);
    const Real one_m[6] = {i == g.gx ? one_x : (Real)1, i == 1 ? one_x : (Real)1,
                           j == g.gy ? one_y : (Real)1, j == 1 ? one_y : (Real)1,
                           k == g.gz ? one_zp : (Real)1, k == 1 ? one_zm : (Real)1};
    const bool interior = i > 1 && i < g.gx && j > 1 && j < g.gy && k > 1 && k < g.gz;
    // diffusion sum: cell_update's expressions
    Real nbsum = 0;
    if (sizeof(Real) == 4) {
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
    const Real cen = oce + nbsum;
    const int br = flags[c];
    Real cl_new, fs_new;
    if (br == BR_RESET || br == BR_NEG) {
        cl_new = cen;
        fs_new = 0;
    } else if (br == BR_KEEP) {
        cl_new = (sizeof(Real) == 8) ? cen * q.k_inv : cen * q.k_inv + q.c0k;
        fs_new = lspfs;
    } else {
        const double Td = temp_cell(p, nullptr, nullptr, c, j, k, ts);
        if (sizeof(Real) == 8) {
            const Real Tcell = (Real)Td;
            Real c_int = q.cinit + q.m_inv * (Tcell - q.Tliq);
            if (p.tip_curv) c_int = q.cinit + q.m_inv * (Tcell - q.Tliq + q.gibbs * (Real)curv[c]);
            Real dce = cen - oce;
            Real dcl = (c_int - conc) * q.D_xt * 2 + dce / (1 - q.km * lspfs);
            Real dfs = (dcl * ((Real)1. - q.km * lspfs) - dce) * q.km_inv / conc;
            cl_new = conc + dcl;
            fs_new = lspfs + dfs;
        } else {
            const Real dT = (Real)(Td - p.Tliq);
            Real c_int = q.m_inv * dT;
            if (p.tip_curv) c_int = q.m_inv * (dT + q.gibbs * (Real)curv[c]);
            const float dce = (float)nbsum;
            const float u = 1.f - (float)q.km * (float)lspfs;
            const float t2 = ((float)c_int - (float)conc) * (2.f * (float)q.D_xt);
            const float dcl = t2 + __fdividef(dce, u);
            const float dfs = __fdividef(t2 * u * (float)q.km_inv, (float)conc + (float)q.cinit);
            cl_new = conc + dcl;
            fs_new = lspfs + dfs;
        }
        if (br == BR_CLAMP) fs_new = 1;
    }
    ce1[c] = cen;
    cl1[c] = cl_new;
    fs1[c] = fs_new;
}

// ----------------------------------------------------------------- adjoint
// Pass A (pointwise).  In:  lce = adjoint of ce after the step, lcl1 = of cl
// after the step.  Out: lce = adjoint of ce before the step, nu = adjoint of
// the cell's diffusion sum.
template <typename Real>
__global__ void __launch_bounds__(ADJ_NT) k_adj_a(Geo g, Phys p, const unsigned char *__restrict__ flags,
                                                  const Real *__restrict__ fs0, Real *__restrict__ lce,
                                                  const Real *__restrict__ lcl1, Real *__restrict__ nu)
{
    int i, j, k;
    long long c;
    if (!interior_cell(g, blockIdx.x * (long long)ADJ_NT + threadIdx.x, i, j, k, c)) return;
    const int br = flags[c];
    const Real a_ce = lce[c], a_cl = lcl1[c];
    Real n, b;
    if (br == BR_RESET || br == BR_NEG) {  // cl' = ce' = oce + nbsum
        n = a_ce + a_cl;
        b = n;
    } else if (br == BR_KEEP) {            // cl' = ce' / k
        n = a_ce + a_cl * (Real)p.k_inv;
        b = n;
    } else {                               // cl' = cl + t2 + nbsum / u
        const Real u = (Real)1 - (Real)p.km * fs0[c];
        n = a_ce + a_cl / u;
        b = a_ce;
    }
    nu[c] = n;
    lce[c] = b;
}

// Parameter-gradient slots accumulated per block by pass B.
enum AdjSlot : int { AS_RL = 0, AS_DXT, AS_KM, AS_KMINV, AS_KINV, AS_GIBBS, AS_COUNT };

// Pass B (gather).  Adjoints of cl and fs before the step, and this step's
// contribution to the parameter gradients (per-block partial sums).
template <typename Real>
__global__ void __launch_bounds__(ADJ_NT) k_adj_b(Geo g, Phys p, const unsigned char *__restrict__ flags,
                                                  const double *__restrict__ curv, const Real *__restrict__ ce0,
                                                  const Real *__restrict__ cl0, const Real *__restrict__ fs0,
                                                  const Real *__restrict__ ce1, const Real *__restrict__ nu,
                                                  const Real *__restrict__ lcl1, const Real *__restrict__ lfs1,
                                                  Real *__restrict__ lcl0, Real *__restrict__ lfs0,
                                                  double *__restrict__ partial, unsigned long long ts)
{
    double acc[AS_COUNT] = {0, 0, 0, 0, 0, 0};
    int i, j, k;
    long long c;
    if (interior_cell(g, blockIdx.x * (long long)ADJ_NT + threadIdx.x, i, j, k, c)) {
        // absolute concentrations (the FP32 form stores ce, cl - Cinit)
        const Real off = (sizeof(Real) == 4) ? (Real)p.cinit : (Real)0;
        const Real rs = (Real)p.rs, rl = (Real)p.rl;
        long long o[6];
        nb_offsets(g, o);
        const Real conc = cl0[c] + off, lspfs = fs0[c];
        const Real nu_c = nu[c];
        const Real one_x = (Real)(1 - g.padx), one_y = (Real)(1 - g.pady), one_zp = (Real)(1 - g.padz_hi),
               one_zm = (Real)(1 - g.padz_lo);
        const Real one_m[6] = {i == g.gx ? one_x : (Real)1, i == 1 ? one_x : (Real)1,
                               j == g.gy ? one_y : (Real)1, j == 1 ? one_y : (Real)1,
                               k == g.gz ? one_zp : (Real)1, k == 1 ? one_zm : (Real)1};
        Real gcl = 0, gfs = 0, grl = 0;
#pragma unroll
        for (int n = 0; n < 6; n++) {
            const long long cn = c + o[n];
            const Real cl_n = cl0[cn] + off, fs_n = fs0[cn];
            const Real fs_av = (Real)0.5 * (lspfs + fs_n);
            const Real r = rs * fs_av + rl * ((Real)1 - fs_av);
            // a neighbour inside the domain sees this cell with factor 1
            const Real nu_n = nb_inside(g, n, i, j, k) ? nu[cn] : (Real)0;
            gcl += nu_n * r - nu_c * r * one_m[n];
            gfs += (Real)0.5 * (rs - rl) * (nu_c * (cl_n - conc) * one_m[n] + nu_n * (conc - cl_n));
            grl += nu_c * ((Real)1 - fs_av) * (cl_n - conc) * one_m[n];
        }
        acc[AS_RL] = (double)grl;
        const int br = flags[c];
        const Real a_cl = lcl1[c], a_fs = lfs1[c];
        if (br == BR_KEEP) {
            gfs += a_fs;                                      // fs' = fs
            acc[AS_KINV] = (double)a_cl * ((double)ce1[c] + (double)off);  // cl' = ce' k_inv
        } else if (br == BR_GROW || br == BR_CLAMP) {
            const Real D_xt = (Real)p.D_xt, km = (Real)p.km, km_inv = (Real)p.km_inv, m_inv = (Real)p.m_inv;
            const double Td = temp_cell(p, nullptr, nullptr, c, j, k, ts);
            const Real kap = p.tip_curv ? (Real)curv[c] : (Real)0;
            const Real c_int = (Real)p.cinit + m_inv * ((Real)(Td - p.Tliq) + (Real)p.gibbs * kap);
            const Real u = (Real)1 - km * lspfs;
            const Real dce = ce1[c] - ce0[c];          // the diffusion sum
            const Real t2 = (c_int - conc) * (Real)2 * D_xt;
            // cl' = cl + t2 + dce / u
            gcl += a_cl * ((Real)1 - (Real)2 * D_xt);
            gfs += a_cl * dce * km / (u * u);
            acc[AS_DXT] += (double)(a_cl * (Real)2 * (c_int - conc));
            acc[AS_KM] += (double)(a_cl * dce * lspfs / (u * u));
            acc[AS_GIBBS] += (double)(a_cl * (Real)2 * D_xt * m_inv * kap);
            if (br == BR_GROW) {
                // fs' = fs + W km_inv / cl with W = dcl u - dce = t2 u
                const Real W = t2 * u;
                gcl += a_fs * km_inv * (-(Real)2 * D_xt * u / conc - W / (conc * conc));
                gfs += a_fs * ((Real)1 - km * t2 * km_inv / conc);
                acc[AS_DXT] += (double)(a_fs * (Real)2 * (c_int - conc) * u * km_inv / conc);
                acc[AS_KM] += (double)(-a_fs * lspfs * t2 * km_inv / conc);
                acc[AS_KMINV] += (double)(a_fs * W / conc);
                acc[AS_GIBBS] += (double)(a_fs * (Real)2 * D_xt * m_inv * kap * u * km_inv / conc);
            }
        }
        lcl0[c] = gcl;
        lfs0[c] = gfs;
    }
    // block sums of the parameter terms, in a fixed order
    __shared__ double sh[AS_COUNT][ADJ_NT / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s < AS_COUNT; s++) {
        double v = acc[s];
        for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
        if (lane == 0) sh[s][w] = v;
    }
    __syncthreads();
    if (threadIdx.x < AS_COUNT) {
        double v = 0;
        for (int q = 0; q < ADJ_NT / 32; q++) v += sh[threadIdx.x][q];
        partial[(long long)blockIdx.x * AS_COUNT + threadIdx.x] = v;
    }
}

// Adds the per-block partials of one step to the running gradient (one
// block; fixed order, so the result is reproducible).
__global__ void k_adj_fold(const double *__restrict__ partial, int nblocks, double *__restrict__ grad)
{
    __shared__ double sh[AS_COUNT][32];
    const int s = threadIdx.y, lane = threadIdx.x;  // blockDim (32, AS_COUNT)
    double v = 0;
    for (int b = lane; b < nblocks; b += 32) v += partial[(long long)b * AS_COUNT + s];
    sh[s][lane] = v;
    __syncthreads();
    if (lane == 0) {
        double t = 0;
        for (int q = 0; q < 32; q++) t += sh[s][q];
        grad[s] += t;
    }
}

// Terminal adjoint of L = 1/2 sum (ce - target)^2 over interior cells:
// lce = ce - target, lcl = lfs = 0; per-block partial sums of the loss.
template <typename Real>
__global__ void __launch_bounds__(ADJ_NT) k_adj_terminal(Geo g, double cinit_off, const Real *__restrict__ ce,
                                                         const double *__restrict__ target, Real *lce, Real *lcl,
                                                         Real *lfs, double *__restrict__ partial)
{
    int i, j, k;
    long long c;
    double l = 0;
    if (interior_cell(g, blockIdx.x * (long long)ADJ_NT + threadIdx.x, i, j, k, c)) {
        const double d = ((double)ce[c] + cinit_off) - target[c];
        l = 0.5 * d * d;
        if (lce) {
            lce[c] = (Real)d;
            lcl[c] = 0;
            lfs[c] = 0;
        }
    }
    __shared__ double sh[ADJ_NT / 32];
    for (int d = 16; d > 0; d >>= 1) l += __shfl_down_sync(0xffffffffu, l, d);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int q = 0; q < ADJ_NT / 32; q++) t += sh[q];
        partial[blockIdx.x] = t;
    }
}

__global__ void k_sum_partials(const double *__restrict__ partial, int n, double *out)
{
    __shared__ double sh[256];
    double v = 0;
    for (int b = threadIdx.x; b < n; b += 256) v += partial[b];
    sh[threadIdx.x] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int q = 0; q < 256; q++) t += sh[q];
        *out = t;
    }
}

// ------------------------------------------------------------------ launchers
static int adj_blocks(const Geo &g) { return (int)(((long long)g.gx * g.gy * g.gz + ADJ_NT - 1) / ADJ_NT); }

int adj_nblocks(const Geo &g) { return adj_blocks(g); }

int launch_replay(const Geo &g, const Phys &p, int precision, const void *const x0[3], void *const x1[3],
                  const unsigned char *flags, const double *curv, unsigned long long ts, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (precision == MMS_PREC_F32)
        k_replay<float><<<adj_blocks(g), ADJ_NT, 0, st>>>(g, p, (const float *)x0[0], (const float *)x0[1],
                                                           (const float *)x0[2], (float *)x1[0], (float *)x1[1],
                                                           (float *)x1[2], flags, curv, ts);
    else
        k_replay<double><<<adj_blocks(g), ADJ_NT, 0, st>>>(g, p, (const double *)x0[0], (const double *)x0[1],
                                                            (const double *)x0[2], (double *)x1[0],
                                                            (double *)x1[1], (double *)x1[2], flags, curv, ts);
    return 1;
}

int launch_adj_step(const Geo &g, const Phys &p, int precision, const void *const x0[3], const void *ce1,
                    const unsigned char *flags, const double *curv, void *lce, const void *lcl1, const void *lfs1,
                    void *lcl0, void *lfs0, void *nu, double *partial, double *grad, unsigned long long ts,
                    void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    const int nb = adj_blocks(g);
    if (precision == MMS_PREC_F32) {
        k_adj_a<float><<<nb, ADJ_NT, 0, st>>>(g, p, flags, (const float *)x0[2], (float *)lce, (const float *)lcl1,
                                               (float *)nu);
        k_adj_b<float><<<nb, ADJ_NT, 0, st>>>(g, p, flags, curv, (const float *)x0[0], (const float *)x0[1],
                                               (const float *)x0[2], (const float *)ce1, (const float *)nu,
                                               (const float *)lcl1, (const float *)lfs1, (float *)lcl0,
                                               (float *)lfs0, partial, ts);
    } else {
        k_adj_a<double><<<nb, ADJ_NT, 0, st>>>(g, p, flags, (const double *)x0[2], (double *)lce,
                                                (const double *)lcl1, (double *)nu);
        k_adj_b<double><<<nb, ADJ_NT, 0, st>>>(g, p, flags, curv, (const double *)x0[0], (const double *)x0[1],
                                                (const double *)x0[2], (const double *)ce1, (const double *)nu,
                                                (const double *)lcl1, (const double *)lfs1, (double *)lcl0,
                                                (double *)lfs0, partial, ts);
    }
    k_adj_fold<<<1, dim3(32, AS_COUNT), 0, st>>>(partial, nb, grad);
    return 3;
}

int launch_adj_terminal(const Geo &g, int precision, double cinit_off, const void *ce, const double *target,
                        void *lce, void *lcl, void *lfs, double *partial, double *loss_out, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    const int nb = adj_blocks(g);
    if (precision == MMS_PREC_F32)
        k_adj_terminal<float><<<nb, ADJ_NT, 0, st>>>(g, cinit_off, (const float *)ce, target, (float *)lce,
                                                      (float *)lcl, (float *)lfs, partial);
    else
        k_adj_terminal<double><<<nb, ADJ_NT, 0, st>>>(g, cinit_off, (const double *)ce, target, (double *)lce,
                                                       (double *)lcl, (double *)lfs, partial);
    k_sum_partials<<<1, 256, 0, st>>>(partial, nb, loss_out);
    return 2;
}

}  // namespace mms
