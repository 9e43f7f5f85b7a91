// ExcludedVolume forces of one system held by the caller in device memory,
// without any device allocation (mjg_exv_force_noalloc in mjolnir_b200.h).
//
// Who needs this: code that runs where cudaMalloc is not available to it --
// inside a host that owns all device memory itself (a framework with its own
// pool, an embedding that forbids allocation after start-up) -- cannot create
// an mjg_context, whose arena is allocated at mjg_commit.  This entry point
// needs nothing but the caller's input and output buffers: the cell list it
// builds lives in a fixed, file-scope device array that every GPU loading the
// library holds until the process exits.
//
// The force is the ExcludedVolume pair sum over all particle pairs within
// sigma_ij * cutoff_ratio (sigma_ij = r_i + r_j), every particle taking part
// and no pair excluded, evaluated in FP64 with the reference's expressions
// (forcefield/global/GlobalPairExcludedVolumeInteraction.hpp:148-195); it is
// the same quantity mjg_term_force returns for MJG_TERM_EXV of a system with
// no ignore rules.  Each particle walks its 27 neighbouring cells (no Verlet
// margin), so its force is written once, without atomics.
#include "../../include/mjolnir_b200.h"
#include "common.cuh"

#include <cstdio>
#include <mutex>

namespace mjg {
namespace {

constexpr int NA_MAX_PARTICLES = 65536;
constexpr int NA_MAX_CELLS     = 65536;
constexpr int NA_TPB           = 256;

// header: [0] dims x, [1] dims y, [2] dims z, [3] hashed, [4..5] max radius (double bits)
struct NaScratch {
    int    header[8];
    double inv_w;
    double pad[7];
    int    count[NA_MAX_CELLS];
    int    start[NA_MAX_CELLS + 1];
    int    fill[NA_MAX_CELLS];
    int    order[NA_MAX_PARTICLES];
};

// The one scratch area of this entry point (about 1 MiB per device).  In host
// code this name is only a stand-in; kernels receive the device address that
// cudaGetSymbolAddress returns.
static __device__ __align__(256) NaScratch g_na_scratch;

struct NaBox {
    int periodic;
    double lower[3], width[3], halfw[3];
};

// one block: largest radius, grid shape, counters to zero
__global__ void k_na_setup(NaScratch* sc, long long n, const double* radius, double cutoff_ratio,
                           NaBox box, double* energy)
{
    __shared__ double red[NA_TPB];
    double m = 0.0;
    for(long long i = threadIdx.x; i < n; i += NA_TPB) {m = fmax(m, radius[i]);}
    red[threadIdx.x] = m;
    __syncthreads();
    for(int o = NA_TPB / 2; o > 0; o >>= 1)
    {
        if(threadIdx.x < o) {red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);}
        __syncthreads();
    }
    if(threadIdx.x == 0)
    {
        const double rc = red[0] * 2 * cutoff_ratio;   // ExcludedVolumePotential::max_cutoff
        int d[3];
        if(box.periodic)
        {
            for(int x = 0; x < 3; ++x)
            {
                const double c = rc > 0 ? floor(box.width[x] / rc) : 3.0;
                d[x] = (int)fmin(fmax(c, 3.0), 64.0);   // at least 3, cells at least rc wide
            }
            while((long long)d[0] * d[1] * d[2] > NA_MAX_CELLS)
            {
                int b = 0;
                for(int x = 1; x < 3; ++x) {if(d[x] > d[b]) {b = x;}}
                d[b] -= 1;
            }
            sc->inv_w = 0.0;
        }
        else
        {
            // unbounded space: cells rc wide hashed modulo a small grid
            int dd = (int)ceil(cbrt((double)n));
            dd = dd < 3 ? 3 : (dd > 32 ? 32 : dd);
            d[0] = d[1] = d[2] = dd;
            sc->inv_w = rc > 0 ? 1.0 / (rc * (1 + 1e-9)) : 0.0;
        }
        sc->header[0] = d[0]; sc->header[1] = d[1]; sc->header[2] = d[2];
        sc->header[3] = box.periodic ? 0 : 1;
        *energy = 0.0;
    }
    // the previous call's contents must not leak into this one
    for(int c = threadIdx.x; c < NA_MAX_CELLS; c += NA_TPB) {sc->count[c] = 0; sc->fill[c] = 0;}
}

__device__ __forceinline__ int na_coord(const NaScratch* sc, const NaBox& box, double x, int axis)
{
    const int d = sc->header[axis];
    if(box.periodic)
    {
        // wrapped: a particle a little outside [lower, upper) lands in the
        // cell its periodic image occupies, next to its image neighbours
        long long c = (long long)floor((x - box.lower[axis]) / (box.width[axis] / d)) % d;
        return (int)(c < 0 ? c + d : c);
    }
    long long c = (long long)floor(x * sc->inv_w) % d;
    return (int)(c < 0 ? c + d : c);
}

__device__ __forceinline__ int na_cell(const NaScratch* sc, int x, int y, int z)
{
    return x + sc->header[0] * (y + sc->header[1] * z);
}

__global__ void k_na_bin(NaScratch* sc, long long n, const double* pos, NaBox box)
{
    const long long i = (long long)blockIdx.x * NA_TPB + threadIdx.x;
    if(i >= n) {return;}
    const int c = na_cell(sc, na_coord(sc, box, pos[3 * i], 0), na_coord(sc, box, pos[3 * i + 1], 1),
                          na_coord(sc, box, pos[3 * i + 2], 2));
    atomicAdd(&sc->count[c], 1);
}

// one block: exclusive scan of the cell counts
__global__ void k_na_scan(NaScratch* sc)
{
    __shared__ int warp_tot[NA_TPB / 32];
    __shared__ int carry;
    const int ncell = sc->header[0] * sc->header[1] * sc->header[2];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if(threadIdx.x == 0) {carry = 0;}
    __syncthreads();
    for(int base = 0; base < ncell; base += NA_TPB)
    {
        const int c = base + threadIdx.x;
        const int v = c < ncell ? sc->count[c] : 0;
        int incl = v;
        for(int o = 1; o < 32; o <<= 1)
        {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if(lane >= o) {incl += y;}
        }
        if(lane == 31) {warp_tot[w] = incl;}
        __syncthreads();
        if(w == 0)
        {
            const int x = lane < NA_TPB / 32 ? warp_tot[lane] : 0;
            int xi = x;
            for(int o = 1; o < 32; o <<= 1)
            {
                const int y = __shfl_up_sync(0xffffffffu, xi, o);
                if(lane >= o) {xi += y;}
            }
            if(lane < NA_TPB / 32) {warp_tot[lane] = xi - x;}
        }
        __syncthreads();
        const int excl = carry + warp_tot[w] + incl - v;
        if(c < ncell) {sc->start[c] = excl;}
        __syncthreads();
        if(threadIdx.x == NA_TPB - 1) {carry = excl + v;}
        __syncthreads();
    }
    if(threadIdx.x == 0) {sc->start[ncell] = carry;}
}

__global__ void k_na_scatter(NaScratch* sc, long long n, const double* pos, NaBox box)
{
    const long long i = (long long)blockIdx.x * NA_TPB + threadIdx.x;
    if(i >= n) {return;}
    const int c = na_cell(sc, na_coord(sc, box, pos[3 * i], 0), na_coord(sc, box, pos[3 * i + 1], 1),
                          na_coord(sc, box, pos[3 * i + 2], 2));
    sc->order[sc->start[c] + atomicAdd(&sc->fill[c], 1)] = (int)i;
}

__global__ void k_na_force(const NaScratch* sc, long long n, const double* pos, const double* radius,
                           double eps, double cutoff_ratio, NaBox box, double* force, double* energy)
{
    const long long i = (long long)blockIdx.x * NA_TPB + threadIdx.x;
    double e = 0.0;
    if(i < n)
    {
        const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2], ri = radius[i];
        const double crsq = cutoff_ratio * cutoff_ratio;
        const double coef_at_cutoff = pow(1.0 / cutoff_ratio, 12);   // ExcludedVolumePotential.hpp:44-48
        const double eps12 = eps * 12;
        const int dx_ = sc->header[0], dy_ = sc->header[1], dz_ = sc->header[2];
        const int cx = na_coord(sc, box, xi, 0), cy = na_coord(sc, box, yi, 1), cz = na_coord(sc, box, zi, 2);
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for(int oz = -1; oz <= 1; ++oz)
        for(int oy = -1; oy <= 1; ++oy)
        for(int ox = -1; ox <= 1; ++ox)
        {
            const int x = (cx + ox + dx_) % dx_, y = (cy + oy + dy_) % dy_, z = (cz + oz + dz_) % dz_;
            const int c = na_cell(sc, x, y, z);
            for(int m = sc->start[c]; m < sc->start[c + 1]; ++m)
            {
                const int j = sc->order[m];
                if(j == i) {continue;}
                double ddx = pos[3 * j] - xi, ddy = pos[3 * j + 1] - yi, ddz = pos[3 * j + 2] - zi;
                if(box.periodic)
                {
                    ddx = min_image(ddx, box.halfw[0], box.width[0]);
                    ddy = min_image(ddy, box.halfw[1], box.width[1]);
                    ddz = min_image(ddz, box.halfw[2], box.width[2]);
                }
                const double l_sq = ddx * ddx + ddy * ddy + ddz * ddz;
                const double sigma = ri + radius[j];
                const double sigma_sq = sigma * sigma;
                if(sigma_sq * crsq < l_sq) {continue;}
                const double rcp = 1.0 / l_sq;
                const double s2 = sigma_sq * rcp;
                const double s6 = s2 * s2 * s2;
                const double cf = -eps12 * s6 * s6 * rcp;
                fx += ddx * cf; fy += ddy * cf; fz += ddz * cf;
                if(i < j) {e += eps * (s6 * s6 - coef_at_cutoff);}
            }
        }
        force[3 * i] = fx; force[3 * i + 1] = fy; force[3 * i + 2] = fz;
    }
    for(int o = 16; o > 0; o >>= 1) {e += __shfl_xor_sync(0xffffffffu, e, o);}
    if((threadIdx.x & 31) == 0 && e != 0.0) {atomicAdd(energy, e);}
}

// Device address of the scratch array, looked up once per CUDA context: the
// address belongs to the context that was current at the lookup, and a device
// reset (cudaDeviceReset, or a host framework resetting the primary context)
// makes a new context in which the array has a new address.  The current
// context is read through the driver's cuCtxGetCurrent, found at run time so
// that the library does not link against the driver.
std::mutex g_na_mutex;
struct NaSlot {
    void* ctx;
    NaScratch* ptr;
};
NaSlot g_na_slots[64] = {};
int g_na_nslots = 0;
using CtxGetCurrent = int (*)(void**);
CtxGetCurrent g_ctx_get_current = nullptr;

// the current context (nullptr when none is current or the driver does not
// say); called with g_na_mutex held
void* current_context()
{
    if(!g_ctx_get_current)
    {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if(cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess ||
           q != cudaDriverEntryPointSuccess || !fn)
        {
            cudaGetLastError();
            return nullptr;
        }
        g_ctx_get_current = reinterpret_cast<CtxGetCurrent>(fn);
    }
    void* ctx = nullptr;
    return g_ctx_get_current(&ctx) == 0 ? ctx : nullptr;
}

}  // namespace
}  // namespace mjg

using namespace mjg;

extern "C" MJG_API int mjg_exv_force_noalloc(int64_t n, int boundary, const double* lower,
                                             const double* upper, const double* pos,
                                             const double* radius, double epsilon,
                                             double cutoff_ratio, double* force, double* energy,
                                             void* stream)
{
    if(n <= 0 || !pos || !radius || !force || !energy || !(cutoff_ratio > 0)) {return MJG_EINVAL;}
    if(n > NA_MAX_PARTICLES)
    {
        std::fprintf(stderr, "mjg_exv_force_noalloc: %lld particles exceed the limit of %d\n",
                     (long long)n, NA_MAX_PARTICLES);
        return MJG_EINVAL;
    }
    if(boundary != MJG_UNLIMITED && boundary != MJG_PERIODIC_CUBOID) {return MJG_EINVAL;}
    NaBox box{};
    box.periodic = boundary == MJG_PERIODIC_CUBOID;
    if(box.periodic)
    {
        if(!lower || !upper) {return MJG_EINVAL;}
        for(int x = 0; x < 3; ++x)
        {
            box.lower[x] = lower[x];
            box.width[x] = upper[x] - lower[x];
            box.halfw[x] = box.width[x] / 2;
            if(!(box.width[x] > 0)) {return MJG_EINVAL;}
        }
    }
    int dev = 0;
    if(cudaGetDevice(&dev) != cudaSuccess || dev < 0) {cudaGetLastError(); return MJG_ECUDA;}
    NaScratch* sc = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_na_mutex);
        // the first call in a context (the first on a device, or the first
        // after a reset) has the runtime make the device's primary context
        // current (cudaSetDevice initialises it), then looks the array's
        // address up in it; without a context handle the address is looked
        // up on every call
        if(cudaSetDevice(dev) != cudaSuccess) {cudaGetLastError(); return MJG_ECUDA;}
        void* ctx = current_context();
        for(int k = 0; k < g_na_nslots && ctx; ++k)
        {
            if(g_na_slots[k].ctx == ctx) {sc = g_na_slots[k].ptr; break;}
        }
        if(!sc)
        {
            void* p = nullptr;
            if(cudaGetSymbolAddress(&p, g_na_scratch) != cudaSuccess || !p)
            {
                cudaGetLastError();
                return MJG_ECUDA;
            }
            sc = static_cast<NaScratch*>(p);
            if(ctx)
            {
                // keep at most 64 contexts; the oldest entry gives way
                if(g_na_nslots < 64) {++g_na_nslots;}
                for(int k = g_na_nslots - 1; k > 0; --k) {g_na_slots[k] = g_na_slots[k - 1];}
                g_na_slots[0] = NaSlot{ctx, sc};
            }
        }
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const unsigned nb = (unsigned)((n + NA_TPB - 1) / NA_TPB);
    k_na_setup  <<<1, NA_TPB, 0, s>>>(sc, n, radius, cutoff_ratio, box, energy);
    k_na_bin    <<<nb, NA_TPB, 0, s>>>(sc, n, pos, box);
    k_na_scan   <<<1, NA_TPB, 0, s>>>(sc);
    k_na_scatter<<<nb, NA_TPB, 0, s>>>(sc, n, pos, box);
    k_na_force  <<<nb, NA_TPB, 0, s>>>(sc, n, pos, radius, epsilon, cutoff_ratio, box, force, energy);
    return cudaGetLastError() == cudaSuccess ? MJG_OK : MJG_ECUDA;
}
