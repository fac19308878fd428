/*
 * fx_calc_dt_noalloc: the CFL timestep reduction of prj_timeint_calc_dt
 * (reference src/prj_timeint.c:2144-2256) over caller-owned device state,
 * with its scratch in a fixed device array instead of allocated memory.
 *
 * Two launches on the caller's stream:
 *   k_dt_partial   one CTA per listed block: min over the block's 16^3 active
 *                  cells of cfl / sum_d (|v_d| + c_s) / dx_d, as an ordered
 *                  integer key, into g_dt_partial[list position]; a listed
 *                  index outside [0, nblocks) reads nothing and stores the
 *                  smallest key, which decodes to NaN;
 *   k_dt_finish    one CTA: min of the nlist keys and the reference's initial
 *                  dt_min = 1e99 (src/prj_timeint.c:2147), times the
 *                  integrator's factor (6 for eSSPRK10_4,
 *                  src/prj_timeint.c:2250-2251), stored as a double at the
 *                  caller's output pointer.
 * Every scratch word k_dt_finish reads was written by k_dt_partial of the
 * same call, so the scratch needs no clearing and nothing carries over from
 * one call to the next.  The per-cell arithmetic is the one the context's
 * k_calc_dt evaluates, in the same order, so both give the same double.
 */
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/fornax_b200.h"
#include "fx_layout.h"
#include "fx_physics.cuh"

namespace {

constexpr int kCells = FX_BS * FX_BS * FX_BS;
constexpr int kPartialThreads = 256;
constexpr int kFinishThreads = 1024;
constexpr int kMaxDevices = 64;

/* one ordered key per listed block: FX_NOALLOC_MAX_BLOCKS * 8 B = 512 KiB */
static __device__ __align__(256) unsigned long long g_dt_partial[FX_NOALLOC_MAX_BLOCKS];

std::mutex g_mu;
unsigned long long *g_partial_addr[kMaxDevices] = {};

__device__ __forceinline__ unsigned long long dt_key(double d)
{
    const unsigned long long bits = (unsigned long long)__double_as_longlong(d);
    return (bits >> 63) ? ~bits : (bits | 0x8000000000000000ULL);
}

__device__ __forceinline__ double dt_from_key(unsigned long long key)
{
    const unsigned long long bits = (key >> 63) ? (key & 0x7fffffffffffffffULL) : ~key;
    return __longlong_as_double((long long)bits);
}

/* min over a CTA; the result is valid in thread 0 */
template <int NT>
__device__ __forceinline__ unsigned long long cta_min(unsigned long long key)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_down_sync(0xffffffffu, key, off);
        key = o < key ? o : key;
    }
    __shared__ unsigned long long smin[NT / 32];
    if ((threadIdx.x & 31) == 0) {
        smin[threadIdx.x >> 5] = key;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 1; q < NT / 32; ++q) {
            key = smin[q] < key ? smin[q] : key;
        }
    }
    return key;
}

__global__ void __launch_bounds__(kPartialThreads) k_dt_partial(const double *__restrict__ W, int nv, int ns,
    const double *__restrict__ dx, int nblocks, const int *__restrict__ blist, double gamma, double cfl,
    unsigned long long *__restrict__ partial)
{
    const int b = blist ? blist[blockIdx.x] : (int)blockIdx.x;
    if (b < 0 || b >= nblocks) {
        if (threadIdx.x == 0) {
            partial[blockIdx.x] = 0ULL; /* decodes to NaN and wins the min */
        }
        return;
    }
    /* stage slot 0 of block b: W + b * nv * ns * NCELLS, variables ns * NCELLS apart */
    const size_t vs = (size_t)ns * FX_NCELLS;
    const double *w = W + (size_t)b * nv * vs;
    const double dx0 = dx[3 * (size_t)b + 0];
    const double dx1 = dx[3 * (size_t)b + 1];
    const double dx2 = dx[3 * (size_t)b + 2];
    unsigned long long key = ~0ULL;
    for (int t = threadIdx.x; t < kCells; t += kPartialThreads) {
        const int k = t % FX_BS;
        const int j = (t / FX_BS) % FX_BS;
        const int i = t / (FX_BS * FX_BS);
        const int c = fx_lidx(i, j, k);
        const double rho = w[FX_RHO * vs + c];
        const double p = fx_pressure(gamma, rho, w[FX_EINT * vs + c]);
        const double cs = sqrt(gamma * p / rho);
        const double denom = (fabs(w[FX_V1 * vs + c]) + cs) / dx0 +
            (fabs(w[FX_V2 * vs + c]) + cs) / dx1 +
            (fabs(w[FX_V3 * vs + c]) + cs) / dx2;
        const double dt_cell = cfl / denom;
        if (dt_cell == dt_cell) {
            const unsigned long long kc = dt_key(dt_cell);
            key = kc < key ? kc : key;
        }
    }
    key = cta_min<kPartialThreads>(key);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = key;
    }
}

__global__ void __launch_bounds__(kFinishThreads) k_dt_finish(const unsigned long long *__restrict__ partial,
    int nlist, double mult, double *__restrict__ dt)
{
    unsigned long long key = threadIdx.x == 0 ? dt_key(1.0e99) : ~0ULL;
    for (int q = threadIdx.x; q < nlist; q += kFinishThreads) {
        key = partial[q] < key ? partial[q] : key;
    }
    key = cta_min<kFinishThreads>(key);
    if (threadIdx.x == 0) {
        *dt = dt_from_key(key) * mult;
    }
}

/* The scratch address of the current device, resolved once per device. */
int partial_scratch(unsigned long long **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return FX_ECUDA;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_partial_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_dt_partial) != cudaSuccess || !p) {
            cudaGetLastError();
            return FX_ECUDA;
        }
        g_partial_addr[dev] = static_cast<unsigned long long *>(p);
    }
    *out = g_partial_addr[dev];
    return FX_SUCCESS;
}

} // namespace

extern "C" int fx_calc_dt_noalloc(const double *W, int mhd, int integrator, const double *dx, int nblocks,
    const int *blocks, int nlist, double gamma, double cfl, void *stream, double *dt)
{
    if (!W || !dx || !dt || nblocks <= 0 || nlist <= 0 || (mhd != 0 && mhd != 1) ||
        (integrator != FX_INT_RK2 && integrator != FX_INT_ESSPRK10_4) || !(gamma > 1.0) || !(cfl > 0.0)) {
        return FX_EINVAL;
    }
    if (nlist > FX_NOALLOC_MAX_BLOCKS) {
        return FX_ETOOBIG;
    }
    /* an error the caller left pending is reported, not consumed */
    if (cudaPeekAtLastError() != cudaSuccess) {
        return FX_ECUDA;
    }
    unsigned long long *partial = nullptr;
    const int rc = partial_scratch(&partial);
    if (rc) {
        return rc;
    }
    const int nv = mhd ? FX_MAXVAR : FX_MAXVAR - 3;
    const int ns = integrator == FX_INT_ESSPRK10_4 ? 3 : 2;
    const double mult = integrator == FX_INT_ESSPRK10_4 ? 6.0 : 1.0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_dt_partial<<<nlist, kPartialThreads, 0, s>>>(W, nv, ns, dx, nblocks, blocks, gamma, cfl, partial);
    if (cudaGetLastError() != cudaSuccess) {
        return FX_ECUDA;
    }
    k_dt_finish<<<1, kFinishThreads, 0, s>>>(partial, nlist, mult, dt);
    if (cudaGetLastError() != cudaSuccess) {
        return FX_ECUDA;
    }
    return FX_SUCCESS;
}
