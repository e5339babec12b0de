// Allocation-free reduction of a caller-owned field: the fraction-solid,
// solid-volume and solute sums of mms_reduce (computeFS loop.c:173-183,
// solid_volume growth.c:971-978, reduce_fs growth.c:541-566), taken over a
// device buffer in the reference's halo'd layout, with every intermediate in
// a fixed device array of this library instead of in memory obtained per call.
//
// Who needs this.  A host loop that checks the fraction solid every few
// steps, between launches on several streams, cannot afford cudaMalloc or
// cudaFree there: both can synchronise the whole device and so stall the
// overlapped work of every other stream.  A caller that has filled HBM with
// its own fields has nothing left to allocate from, and one that keeps its
// fields in its own pool (a caching allocator, a fixed arena) wants no
// second owner of device memory.  Those callers pass their field and a
// device result slot, and this code touches nothing else.
//
// Limits.  Partial sums of one call live in `na_scratch`, 65536 blocks of
// 16384 interior cells each: at most 2^30 interior cells (1024^3) per call.
// Larger grids are rejected with MMS_ERR_SCRATCH_LIMIT before any device work.
// Calls whose kernels may run at the same time on one device (different
// streams without ordering, or different host threads) share that array and
// race; calls on one stream are ordered and safe.
//
// Set-up.  The array's device address is looked up on the first call made
// with a device current, and kept together with the CUDA context it belongs
// to; a call that finds another context current on that device (after a
// primary-context reset, or under a driver-API context the caller made
// current) looks the address up again in that context.  The first call in a
// context should come before any stream capture in it.
//
// Errors.  The kernels are launched with cudaLaunchKernel and its return
// code is checked, so a pending (non-sticky) error of the caller's own CUDA
// work is neither cleared nor reported as this call's.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../include/mms.h"

namespace {

constexpr int NA_NT = 256;                     // threads per partial-sum block
constexpr long long NA_CELLS_PER_BLOCK = 16384;  // 64 cells per thread
constexpr int NA_MAX_BLOCKS = 65536;           // 2 doubles each: 1 MiB of scratch
constexpr int NA_FIN_NT = 1024;                // one finishing block
constexpr int NA_MAX_DEVICES = 64;

// Per-block (sum, compensation) pairs.  Every slot that the finishing kernel
// reads is written by the first kernel of the same call, so no part of this
// array has to start at zero.
static __device__ __align__(256) double na_scratch[2 * NA_MAX_BLOCKS];

std::mutex na_mu;
// Per device: the id of the context the address was looked up in (CUDA
// context ids are unique for the life of the process, so a context made
// after a reset never matches an older one), and the address.
unsigned long long na_ctxid[NA_MAX_DEVICES];  // zero-initialised: not looked up yet
double *na_addr[NA_MAX_DEVICES];

typedef CUresult (*ctx_get_current_fn)(CUcontext *);
typedef CUresult (*ctx_get_id_fn)(CUcontext, unsigned long long *);

// A driver function through the runtime's driver entry point (the library
// does not link libcuda directly).  Null when the driver does not offer it.
void *driver_fn(const char *name)
{
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
        return nullptr;
    return p;
}

// Id of the context current on the calling thread; 0 if none is current or
// the driver cannot say.
unsigned long long current_context_id()
{
    static ctx_get_current_fn get = (ctx_get_current_fn)driver_fn("cuCtxGetCurrent");
    static ctx_get_id_fn get_id = (ctx_get_id_fn)driver_fn("cuCtxGetId");
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (!get || !get_id || get(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Sum of (s, c) pairs with the error of each addition carried in c
// (Knuth's TwoSum), so the result does not depend on the field's size.
__device__ __forceinline__ void two_sum_add(double &s, double &c, double x)
{
    double t = s + x;
    double bp = t - s;
    c += (s - (t - bp)) + (x - bp);
    s = t;
}

template <typename T>
__global__ void __launch_bounds__(NA_NT) k_reduce_na_partials(const T *__restrict__ f, int gx, int gy,
                                                               long long n, int clamp,
                                                               double *__restrict__ partial)
{
    const long long sy = gx + 2, sz = sy * (gy + 2);
    const long long v0 = blockIdx.x * NA_CELLS_PER_BLOCK;
    const long long v1 = (v0 + NA_CELLS_PER_BLOCK < n) ? v0 + NA_CELLS_PER_BLOCK : n;
    double s = 0.0, c = 0.0;
    for (long long v = v0 + threadIdx.x; v < v1; v += NA_NT) {
        long long i = v % gx, r = v / gx;
        long long j = r % gy, k = r / gy;
        double x = (double)f[(k + 1) * sz + (j + 1) * sy + (i + 1)];
        if (clamp) x = (1.0 < x) ? 1.0 : x;   // min(1, fs), reduce_fs
        two_sum_add(s, c, x);
    }
    __shared__ double ss[NA_NT], sc[NA_NT];
    ss[threadIdx.x] = s;
    sc[threadIdx.x] = c;
    __syncthreads();
    for (int w = NA_NT / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            double a = ss[threadIdx.x], b = sc[threadIdx.x] + sc[threadIdx.x + w];
            two_sum_add(a, b, ss[threadIdx.x + w]);
            ss[threadIdx.x] = a;
            sc[threadIdx.x] = b;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = ss[0];
        partial[2 * blockIdx.x + 1] = sc[0];
    }
}

// Folds the per-block pairs in a fixed order and applies the scaling of the
// requested reduction: CE_SUM s, SOLID_VOLUME s*dx^3, FS_FRACTION
// (s*dx^3)/(ncells*dx^3) as computeFS writes it.
__global__ void __launch_bounds__(NA_FIN_NT) k_reduce_na_finish(const double *__restrict__ partial,
                                                                int nblocks, int what, double vol,
                                                                double ncells, double *out)
{
    double s = 0.0, c = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += NA_FIN_NT) {
        two_sum_add(s, c, partial[2 * b]);
        c += partial[2 * b + 1];
    }
    __shared__ double ss[NA_FIN_NT], sc[NA_FIN_NT];
    ss[threadIdx.x] = s;
    sc[threadIdx.x] = c;
    __syncthreads();
    for (int w = NA_FIN_NT / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            double a = ss[threadIdx.x], e = sc[threadIdx.x] + sc[threadIdx.x + w];
            two_sum_add(a, e, ss[threadIdx.x + w]);
            ss[threadIdx.x] = a;
            sc[threadIdx.x] = e;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double r = ss[0] + sc[0];
        if (what == MMS_REDUCE_SOLID_VOLUME) r = r * vol;
        else if (what == MMS_REDUCE_FS_FRACTION) r = (r * vol) / (ncells * vol);
        *out = r;
    }
}

// Device address of na_scratch in the context current on device `dev`:
// looked up on first use, and again whenever another context is current.
double *scratch_for(int dev)
{
    std::lock_guard<std::mutex> lock(na_mu);
    const unsigned long long id = current_context_id();
    if (!na_addr[dev] || !id || id != na_ctxid[dev]) {
        void *p = nullptr;
        // makes the device's primary context current if no context is
        if (cudaGetSymbolAddress(&p, na_scratch) != cudaSuccess || !p) return nullptr;
        na_addr[dev] = (double *)p;
        na_ctxid[dev] = current_context_id();
    }
    return na_addr[dev];
}

}  // namespace

extern "C" mms_status mms_reduce_field_noalloc(const void *field, mms_precision dtype, int gdimx,
                                               int gdimy, int gdimz, mms_reduction what,
                                               double cell_size, double *out, void *cuda_stream)
{
    if (!field || !out || gdimx <= 0 || gdimy <= 0 || gdimz <= 0) return MMS_ERR_ARG;
    if (dtype != MMS_PREC_F64 && dtype != MMS_PREC_F32) return MMS_ERR_ARG;
    if (what != MMS_REDUCE_FS_FRACTION && what != MMS_REDUCE_SOLID_VOLUME && what != MMS_REDUCE_CE_SUM)
        return MMS_ERR_ARG;
    const long long n = (long long)gdimx * gdimy * gdimz;
    const long long nb = (n + NA_CELLS_PER_BLOCK - 1) / NA_CELLS_PER_BLOCK;
    if (nb > NA_MAX_BLOCKS) return MMS_ERR_SCRATCH_LIMIT;

    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return MMS_ERR_NO_DEVICE;
    if (dev < 0 || dev >= NA_MAX_DEVICES) return MMS_ERR_ARG;
    double *partial = scratch_for(dev);
    if (!partial) return MMS_ERR_CUDA;

    cudaStream_t st = (cudaStream_t)cuda_stream;
    int clamp = (what != MMS_REDUCE_CE_SUM), gx = gdimx, gy = gdimy, nblocks = (int)nb, w = (int)what;
    long long ncell = n;
    const void *fld = field;
    void *pa[] = {(void *)&fld, &gx, &gy, &ncell, &clamp, &partial};
    const void *k1 = (dtype == MMS_PREC_F64) ? (const void *)k_reduce_na_partials<double>
                                             : (const void *)k_reduce_na_partials<float>;
    if (cudaLaunchKernel(k1, dim3((unsigned)nb), dim3(NA_NT), pa, 0, st) != cudaSuccess) return MMS_ERR_CUDA;
    double vol = std::pow(cell_size, 3.0), dn = (double)n;
    void *fa[] = {&partial, &nblocks, &w, &vol, &dn, &out};
    if (cudaLaunchKernel((const void *)k_reduce_na_finish, dim3(1), dim3(NA_FIN_NT), fa, 0, st) != cudaSuccess)
        return MMS_ERR_CUDA;
    return MMS_OK;
}
