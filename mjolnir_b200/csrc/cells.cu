// Cell-list rebuild of the Verlet lists by counting sort and prefix scan.
//
// Replaces PeriodicGridCellList::make / UnlimitedGridCellList::make
// (core/PeriodicGridCellList.hpp:198-351, core/UnlimitedGridCellList.hpp
// :152-255) for every system of the arena that reduce_margin flagged:
//   1. zero the flagged systems' cell counters,
//   2. bin their participants (one atomic increment per participant),
//   3. exclusive scan over all cells of the term (3-phase, 2048 cells/block),
//   4. scatter participants into cell order, sort each cell by participant,
//   5. renumber: slot = position in cell order (spatially coherent slots),
//   6. build each slot's partner list from the 27 neighbouring cells with the
//      reference's membership test, evaluated in FP64 without contraction:
//      has_interaction (i < j of a leading participant, not excluded) and
//      |adjust_direction(r_i, r_j)|^2 < (cutoff (1 + margin))^2.
// The lists hold both directions of every pair (full lists); a pair (a, b) is
// present iff the reference's half list holds (min(a,b), max(a,b)).
#include "kernels.cuh"

namespace mjg {

namespace {

constexpr int TPB = 256;
constexpr int SCAN_TPB = 1024;
constexpr int SCAN_PER_BLOCK = 2 * SCAN_TPB;

__device__ __forceinline__ bool flagged(const Arena& a, int sys, int g)
{
    return a.sys[sys].g[g].rebuild != 0;
}

__global__ void k_cells_zero(Arena a, int g, TermArrays t, const int* cell_sys)
{
    if(*t.any_rebuild == 0) {return;}
    const int c = blockIdx.x * TPB + threadIdx.x;
    if(c >= t.ncell) {return;}
    if(!flagged(a, cell_sys[c], g)) {return;}
    t.cell_count[c] = 0;
    t.cell_fill[c]  = 0;
}

__global__ void k_cells_assign(Arena a, int g, TermArrays t)
{
    if(*t.any_rebuild == 0) {return;}
    const long long p = (long long)blockIdx.x * TPB + threadIdx.x;
    if(p >= t.np) {return;}
    const int s = t.part_sys[p];
    const GlobalParams& G = a.sys[s].g[g];
    if(!G.rebuild) {return;}
    const double4 r = a.pos[t.part_particle[p]];
    const int cx = cell_coord(r.x, G, 0);
    const int cy = cell_coord(r.y, G, 1);
    const int cz = cell_coord(r.z, G, 2);
    const int c = G.cell_off + cx + G.dims[0] * (cy + G.dims[1] * cz);
    t.part_cell[p] = c;
    atomicAdd(&t.cell_count[c], 1);
}

// phase 1: per-block exclusive scan of cell_count into cell_start
__global__ void __launch_bounds__(SCAN_TPB) k_scan_local(TermArrays t)
{
    if(*t.any_rebuild == 0) {return;}
    __shared__ int warp_tot[SCAN_TPB / 32];
    const int base = blockIdx.x * SCAN_PER_BLOCK;
    const int c0 = base + 2 * threadIdx.x;
    const int v0 = c0     < t.ncell ? t.cell_count[c0]     : 0;
    const int v1 = c0 + 1 < t.ncell ? t.cell_count[c0 + 1] : 0;
    const int sum = v0 + v1;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int incl = sum;
#pragma unroll
    for(int o = 1; o < 32; o <<= 1)
    {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if(lane >= o) {incl += y;}
    }
    if(lane == 31) {warp_tot[w] = incl;}
    __syncthreads();
    if(w == 0)
    {
        int x = warp_tot[lane];
        int xi = x;
#pragma unroll
        for(int o = 1; o < 32; o <<= 1)
        {
            const int y = __shfl_up_sync(0xffffffffu, xi, o);
            if(lane >= o) {xi += y;}
        }
        warp_tot[lane] = xi - x;       // exclusive warp offsets
    }
    __syncthreads();
    const int excl = incl - sum + warp_tot[w];
    if(c0     < t.ncell) {t.cell_start[c0]     = excl;}
    if(c0 + 1 < t.ncell) {t.cell_start[c0 + 1] = excl + v0;}
    if(threadIdx.x == SCAN_TPB - 1) {t.block_sums[blockIdx.x] = excl + sum;}
}

// phase 2: exclusive scan of the block totals (one block, serial chunks)
__global__ void __launch_bounds__(SCAN_TPB) k_scan_blocks(TermArrays t, int nblocks)
{
    if(*t.any_rebuild == 0) {return;}
    __shared__ int warp_tot[SCAN_TPB / 32];
    __shared__ int carry;
    if(threadIdx.x == 0) {carry = 0;}
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for(int base = 0; base < nblocks; base += SCAN_TPB)
    {
        const int b = base + threadIdx.x;
        const int v = b < nblocks ? t.block_sums[b] : 0;
        int incl = v;
#pragma unroll
        for(int o = 1; o < 32; o <<= 1)
        {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if(lane >= o) {incl += y;}
        }
        if(lane == 31) {warp_tot[w] = incl;}
        __syncthreads();
        if(w == 0)
        {
            const int x = warp_tot[lane];
            int xi = x;
#pragma unroll
            for(int o = 1; o < 32; o <<= 1)
            {
                const int y = __shfl_up_sync(0xffffffffu, xi, o);
                if(lane >= o) {xi += y;}
            }
            warp_tot[lane] = xi - x;
        }
        __syncthreads();
        const int excl = incl - v + warp_tot[w] + carry;
        __syncthreads();
        if(b < nblocks) {t.block_sums[b] = excl;}
        if(threadIdx.x == SCAN_TPB - 1) {carry = excl + v;}
        __syncthreads();
    }
    if(threadIdx.x == 0) {t.cell_start[t.ncell] = carry;}
}

// phase 3: add block offsets
__global__ void k_scan_add(TermArrays t)
{
    if(*t.any_rebuild == 0) {return;}
    const int c = blockIdx.x * TPB + threadIdx.x;
    if(c >= t.ncell) {return;}
    t.cell_start[c] += t.block_sums[c / SCAN_PER_BLOCK];
}

__global__ void k_cells_scatter(Arena a, int g, TermArrays t, int* slot_tmp)
{
    if(*t.any_rebuild == 0) {return;}
    const long long p = (long long)blockIdx.x * TPB + threadIdx.x;
    if(p >= t.np) {return;}
    if(!flagged(a, t.part_sys[p], g)) {return;}
    const int c = t.part_cell[p];
    const int k = atomicAdd(&t.cell_fill[c], 1);
    slot_tmp[t.cell_start[c] + k] = (int)p;
}

// one warp per cell: rank sort of the members by participant index, so that
// slot order depends only on the cell assignment
__global__ void k_cells_sort(Arena a, int g, TermArrays t, const int* cell_sys, const int* slot_tmp)
{
    if(*t.any_rebuild == 0) {return;}
    const int c = (blockIdx.x * TPB + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if(c >= t.ncell) {return;}
    if(!flagged(a, cell_sys[c], g)) {return;}
    const int b = t.cell_start[c], m = t.cell_start[c + 1] - b;
    for(int e = lane; e < m; e += 32)
    {
        const int v = slot_tmp[b + e];
        int rank = 0;
        for(int u = 0; u < m; ++u) {rank += slot_tmp[b + u] < v ? 1 : 0;}
        t.slot_part[b + rank] = v;
    }
}

__global__ void k_slots_setup(Arena a, int g, TermArrays t)
{
    if(*t.any_rebuild == 0) {return;}
    const long long s = (long long)blockIdx.x * TPB + threadIdx.x;
    if(s >= t.np) {return;}
    const int p = t.slot_part[s];
    const int sys = t.part_sys[p];
    if(!flagged(a, sys, g)) {return;}
    t.slot_particle[s] = t.part_particle[p];
    t.slot_lead[s]     = t.part_lead[p];
    t.slot_sys[s]      = sys;
    t.slot_pd[s].w     = t.part_p0[p];
    if(t.part_p1) {t.slot_p1[s] = t.part_p1[p];}
}

__device__ __forceinline__ bool is_excluded(const Arena& a, int g, int ignore_mol, int i, int j)
{
    if(ignore_mol == IGN_SELF   && a.mol[i] == a.mol[j]) {return true;}
    if(ignore_mol == IGN_OTHERS && a.mol[i] != a.mol[j]) {return true;}
    const long long b = a.ex_start[g][i], e = a.ex_start[g][i + 1];
    for(long long q = b; q < e; ++q)
    {
        const int x = a.ex_idx[g][q];
        if(x > j) {break;}
        if(x == j) {return true;}
    }
    return false;
}

__global__ void __launch_bounds__(TPB) k_build_list(Arena a, int g, TermArrays t)
{
    if(*t.any_rebuild == 0) {return;}
    const long long s = (long long)blockIdx.x * TPB + threadIdx.x;
    if(s >= t.np) {return;}
    const int sys = t.slot_sys[s];
    const SysDev& S = a.sys[sys];
    const GlobalParams& G = S.g[g];
    if(!G.rebuild) {return;}

    const int i = t.slot_particle[s];
    const bool lead_i = t.slot_lead[s] != 0;
    const double4 ri = a.pos[i];
    const int cx = cell_coord(ri.x, G, 0);
    const int cy = cell_coord(ri.y, G, 1);
    const int cz = cell_coord(ri.z, G, 2);
    const bool periodic = S.boundary == B_PERIODIC;
    const int dx_ = G.dims[0], dy_ = G.dims[1], dz_ = G.dims[2];
    const bool wrap = periodic || G.hashed;
    const int cap = t.cap;
    const long long np = t.np;
    int count = 0;

    for(int oz = -1; oz <= 1; ++oz)
    for(int oy = -1; oy <= 1; ++oy)
    for(int ox = -1; ox <= 1; ++ox)
    {
        int x = cx + ox, y = cy + oy, z = cz + oz;
        if(wrap)
        {
            x = x < 0 ? x + dx_ : (x >= dx_ ? x - dx_ : x);
            y = y < 0 ? y + dy_ : (y >= dy_ ? y - dy_ : y);
            z = z < 0 ? z + dz_ : (z >= dz_ ? z - dz_ : z);
        }
        else if(x < 0 || y < 0 || z < 0 || x >= dx_ || y >= dy_ || z >= dz_) {continue;}
        const int c = G.cell_off + x + dx_ * (y + dy_ * z);
        const int b = t.cell_start[c], e = t.cell_start[c + 1];
        for(int q = b; q < e; ++q)
        {
            const int j = t.slot_particle[q];
            if(j == i) {continue;}
            const bool lead_lo = (i < j) ? lead_i : (t.slot_lead[q] != 0);
            if(!lead_lo) {continue;}
            if(is_excluded(a, g, G.ignore_mol, i < j ? i : j, i < j ? j : i)) {continue;}
            const double4 rj = a.pos[j];
            double ddx = __dsub_rn(rj.x, ri.x);
            double ddy = __dsub_rn(rj.y, ri.y);
            double ddz = __dsub_rn(rj.z, ri.z);
            if(periodic)
            {
                ddx = min_image(ddx, S.halfw[0], S.width[0]);
                ddy = min_image(ddy, S.halfw[1], S.width[1]);
                ddz = min_image(ddz, S.halfw[2], S.width[2]);
            }
            const double l2 = __dadd_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)), __dmul_rn(ddz, ddz));
            if(l2 < G.rl2)
            {
                if(count < cap) {t.nbr[(long long)count * np + s] = q;}
                ++count;
            }
        }
    }
    t.nnb[s] = count < cap ? count : cap;
    atomicMax(t.max_count, count);
    if(count > cap) {atomicOr(&a.sys[sys].status, ST_LIST_OVERFLOW);}
}

__global__ void k_rebuild_done(Arena a, int g, TermArrays t, int forced)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if(s < a.nsys)
    {
        GlobalParams& G = a.sys[s].g[g];
        if(G.on && G.rebuild)
        {
            G.rebuild = 0;
            G.current_margin = __dmul_rn(G.cutoff, G.margin);   // ...GridCellList::make, last line
            if(!forced) {G.rebuilds += 1;}   // count only reduce_margin rebuilds
        }
    }
}

__global__ void k_clear_any(TermArrays t) {*t.any_rebuild = 0;}

__global__ void k_force_all(Arena a, int g, TermArrays t)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if(s < a.nsys && a.sys[s].g[g].on) {a.sys[s].g[g].rebuild = 1;}
    if(s == 0) {*t.any_rebuild = 1;}
}

inline unsigned blocks(long long n, int tpb = TPB) {return (unsigned)((n + tpb - 1) / tpb);}

}  // namespace

// cell_sys is stored right behind block_sums (see the context's allocation)
void launch_rebuild(const Arena& a, int g, TermArrays& t, int force_all, cudaStream_t s)
{
    if(!t.on || t.np == 0) {return;}
    const int nblocks = (t.ncell + SCAN_PER_BLOCK - 1) / SCAN_PER_BLOCK;
    const int* cell_sys = t.block_sums + nblocks + 1;
    if(force_all) {k_force_all<<<blocks(a.nsys, 128), 128, 0, s>>>(a, g, t); note_launches(1);}
    k_cells_zero  <<<blocks(t.ncell), TPB, 0, s>>>(a, g, t, cell_sys);
    k_cells_assign<<<blocks(t.np), TPB, 0, s>>>(a, g, t);
    k_scan_local  <<<nblocks, SCAN_TPB, 0, s>>>(t);
    k_scan_blocks <<<1, SCAN_TPB, 0, s>>>(t, nblocks);
    k_scan_add    <<<blocks(t.ncell), TPB, 0, s>>>(t);
    k_cells_scatter<<<blocks(t.np), TPB, 0, s>>>(a, g, t, t.slot_particle);
    k_cells_sort  <<<blocks((long long)t.ncell * 32), TPB, 0, s>>>(a, g, t, cell_sys, t.slot_particle);
    k_slots_setup <<<blocks(t.np), TPB, 0, s>>>(a, g, t);
    k_build_list  <<<blocks(t.np), TPB, 0, s>>>(a, g, t);
    k_rebuild_done<<<blocks(a.nsys, 128), 128, 0, s>>>(a, g, t, force_all);
    k_clear_any   <<<1, 1, 0, s>>>(t);
    note_launches(11);
}

}  // namespace mjg
