// device_common.cuh — device helpers shared by the step kernels (kernels.cu)
// and the adjoint (adjoint.cu).  Both are compiled with -fmad=false, so an
// expression written here rounds the same way in either file.
#pragma once

#include "mms_internal.h"

namespace mms {

// A step stops at the first kernel that sees the stall flag.
__device__ __forceinline__ bool stalled(const Ctl *c)
{
    return *((volatile const int *)&c->stall) != 0;
}

__device__ __forceinline__ void raise_error(Ctl *c, int status)
{
    atomicCAS(&c->status, 0, status);
    atomicExch(&c->stall, (int)STALL_ERROR);
}

// Index check of the bounds-checked build (compiled with -DMMS_BOUNDS): an
// index outside [0, n) raises MMS_ERR_BOUNDS (the step stops at its next
// kernel) and the caller skips the access.  The ordinary build compiles the
// check out.
__device__ __forceinline__ bool in_bounds(Ctl *c, long long i, long long n)
{
#ifdef MMS_BOUNDS
    if ((unsigned long long)i < (unsigned long long)n) return true;
    raise_error(c, MMS_ERR_BOUNDS);
    return false;
#else
    (void)c;
    (void)i;
    (void)n;
    return true;
#endif
}


// direct_temp_calc (temperature.c:24-61) for the analytic models; the AM
// quadrature is precomputed into an array by k_temp_am.  K is the local
// plane; p.kz0 places a slab's planes in the whole domain.
__device__ __forceinline__ double temp_cell(const Phys &p, const double *Tarr, const float *T32, long long cell,
                                            long long J, long long K, unsigned long long ts)
{
    if (p.temp_mode == 2) return T32 ? (double)T32[cell] : Tarr[cell];
    double sim_time = (double)ts * p.ts_delt;
    if (p.temp_mode == 0) return p.T0 - sim_time * p.cool_rate;
    double ry = p.origin[1] + ((double)(int)J + 0.5) * p.cellSize;
    double rz = p.origin[2] + ((double)((int)K + p.kz0) + 0.5) * p.cellSize;
    double axis = (p.gz_is_one ? ry : rz) - p.cellSize * 0.5;
    double tgrad = p.gradient + p.grad_coef * sim_time;
    double v = p.velocity + p.velo_coef * sim_time;
    double vt = 0.5 * (v + p.velocity) * sim_time;
    return p.T0 + tgrad * (axis - vt);
}

// Physics constants in the stencil's arithmetic type.
template <typename Real>
struct PhysR {
    Real rs, rl, liq_slope, k_inv, km, km_inv, m_inv, D_xt, cinit, Tliq, gibbs, c0k;
    // FP32 form: the liquidus rounded down to FP32, and as an FP32 head and
    // the FP32 rounding of its remainder (FP32 temperature arrays)
    float tliq_rd, tliq_h, tliq_l;
};

template <typename Real>
__device__ __forceinline__ PhysR<Real> phys_r(const Phys &p)
{
    PhysR<Real> q;
    q.rs = (Real)p.rs;
    q.rl = (Real)p.rl;
    q.liq_slope = (Real)p.liq_slope;
    q.k_inv = (Real)p.k_inv;
    q.km = (Real)p.km;
    q.km_inv = (Real)p.km_inv;
    q.m_inv = (Real)p.m_inv;
    q.D_xt = (Real)p.D_xt;
    q.cinit = (Real)p.cinit;
    q.Tliq = (Real)p.Tliq;
    q.gibbs = (Real)p.gibbs;
    q.c0k = (Real)(p.cinit * (p.k_inv - 1.0));
    q.tliq_rd = __double2float_rd(p.Tliq);
    q.tliq_h = (float)p.Tliq;
    q.tliq_l = (float)(p.Tliq - (double)q.tliq_h);
    return q;
}

// AM moving-source quadrature: nodes, and the source position and prefactor
// of a step (direct_temp_calc thermal_ana == 1, temperature.c:62-123)
constexpr int AM_NT = 400;

// The FP32 form's tensor-core operand buffer (a.d.am_ximg): the X image of
// am_tc.cu (2^14 X as FP16 head and remainder: [x tile of 128][K-step of 16
// nodes][head, remainder][128 x 16 halves]), then Y and Z with the 400 nodes
// contiguous for each row (YT[J][i], ZT[K][i], FP32), then the B image (the
// scaled products Y Z as FP16 head and remainder: [block of N (y, z)
// rows][K-step][head, remainder][N x 16 halves], N the contraction's tile
// height, room for any N up to 256).  Sizes in floats.
__host__ __device__ constexpr long long am_ximg_part(int gx)
{
    return (long long)((gx + 127) / 128) * (AM_NT / 16) * 2 * (128 * 16) / 2;
}

__host__ __device__ inline float *am_yt(float *img, int gx) { return img + am_ximg_part(gx); }
__host__ __device__ inline float *am_zt(float *img, int gx, int gy)
{
    return img + am_ximg_part(gx) + (long long)(gy + 2) * AM_NT;
}
__host__ __device__ inline unsigned char *am_bimg(float *img, int gx, int gy, int gz)
{
    return (unsigned char *)(img + am_ximg_part(gx) + (long long)(gy + gz + 4) * AM_NT);
}
// 2 x 2 bytes per node and row: one float per node and row
__host__ __device__ constexpr long long am_bimg_part(int gy, int gz)
{
    return ((long long)(gy + 2) * (gz + 2) + 255) * AM_NT;
}

// The step the AM tables (k_am_tables: X, Y, Z, then the per-plane flags
// zon[nz]) were last built for, kept in the table buffer after the flags.
__device__ __forceinline__ unsigned long long *am_tab_step(const int *zon, int nz)
{
    return (unsigned long long *)(((unsigned long long)(zon + nz) + 7ULL) & ~7ULL);
}
// FP32 form: the scale of the B operand (am_b_scale) of the step the tables
// were built for, after the step marker (the FP32 tables leave the room)
__device__ __forceinline__ float *am_tab_sb(const int *zon, int nz) { return (float *)(am_tab_step(zon, nz) + 1); }

struct AmStep {
    double xnow, ynow, znow, lalpha, ls, ldt, Tfront, liniT;
};

__device__ __forceinline__ AmStep am_step(const Phys &p, const AmParams &m, unsigned long long ts)
{
    AmStep s;
    const double sim_time = (double)ts * p.ts_delt;
    const double invlv = 1. / m.lv;
    s.ls = m.lsd / (2. * 1.414);
    double xlen = m.nsbx_times_sbx * p.cellSize;
    xlen = xlen + m.lsd;
    double tline = xlen * invlv;
    const double tpause = 1.5e-4 * invlv;
    tline = tline + tpause;
    double trackno = 0;
    if (m.amtracks > 1) trackno = floor(sim_time / tline);
    s.xnow = m.x0 + (sim_time - trackno * tline) * m.lv;
    s.ynow = m.y0 + trackno * m.lhs;
    s.znow = m.z0;
    s.lalpha = m.lthcon / m.rho_cp;
    const double tsteady = 20 * s.lalpha * invlv * invlv;
    s.ldt = tsteady / AM_NT;
    const double pw = (sim_time < 1e-4) ? 0.0 : m.lpow;
    s.Tfront = m.lab * pw * s.lalpha / (5.568328 * m.lthcon);
    s.liniT = m.liniT;
    return s;
}

// The power of two that scales the products Y_i(y) Z_i(z) into FP16's range
// for the tensor cores: Y <= 1, and Z_i <= ldt / Tl_i <= ldt / Tl_0 (Tl_i =
// sqrt(alpha t_i) (s^2 + 4 alpha t_i) grows with t_i), so the largest
// product is at most ldt / Tl_0, which the scale maps to at most 2^14.
// Subnormal FP16 values keep an absolute resolution of 2^-24, 2^-38 of that
// maximum, so no per-row scale is needed.
__device__ __forceinline__ double am_b_scale(const AmStep &s)
{
    const double lt0 = 0.5 * s.ldt;
    const double zb = s.ldt / (sqrt(s.lalpha * lt0) * (s.ls * s.ls + 4. * s.lalpha * lt0));
    if (!(zb > 0.0) || !(zb < 1e300)) return 1.0;
    return exp2(14.0 - ceil(log2(zb)));
}

}  // namespace mms
