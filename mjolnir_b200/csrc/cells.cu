// Cell-list rebuild of the Verlet lists by counting sort and prefix scan.
//
// Replaces PeriodicGridCellList::make / UnlimitedGridCellList::make
// (core/PeriodicGridCellList.hpp:198-351, core/UnlimitedGridCellList.hpp
// :152-255) for every system of the arena that reduce_margin flagged.  A
// planning kernel turns the flagged systems into a work list of 256-item
// chunks (participants and cells); every later kernel is a persistent grid
// that walks only those chunks, so a step in which 5 of 256 systems rebuild
// costs 5 systems' worth of work:
//   1. zero the flagged systems' cell counters,
//   2. bin their participants (one atomic increment per participant),
//   3. exclusive scan of each flagged system's cells (one block per system),
//   4. scatter participants into cell order, sort each cell by participant,
//   5. renumber: slot = position in cell order (spatially coherent slots),
//   6. build each slot's partner list from the 27 neighbouring cells (one
//      warp per slot) with the reference's membership test, evaluated in FP64
//      without contraction:
//      has_interaction (i < j of a leading participant, not excluded) and
//      |adjust_direction(r_i, r_j)|^2 < (cutoff (1 + margin))^2.
// The lists hold both directions of every pair (full lists); a pair (a, b) is
// present iff the reference's half list holds (min(a,b), max(a,b)).
#include "kernels.cuh"

namespace mjg {

namespace {

constexpr int TPB = 256;
constexpr int CHUNK = 256;          // items per work chunk
constexpr int GRID = 148 * 8;       // persistent grid: 8 blocks of 256 per SM
constexpr int SCAN_TPB = 1024;

// work counters in t.work: [0] participant chunks, [1] cell chunks, [2] flagged systems

__global__ void k_plan(Arena a, int g, TermArrays t, int force_all)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if(s >= a.nsys) {return;}
    GlobalParams& G = a.sys[s].g[g];
    if(!G.on) {return;}
    if(force_all) {G.rebuild = 1;}
    if(!G.rebuild) {return;}
    const int np = (G.nslot + CHUNK - 1) / CHUNK;
    const int nc = (G.ncell + CHUNK - 1) / CHUNK;
    const int bp = atomicAdd(&t.work[0], np);
    const int bc = atomicAdd(&t.work[1], nc);
    t.flagged[atomicAdd(&t.work[2], 1)] = s;
    for(int k = 0; k < np; ++k)
    {
        const int b = G.slot_off + k * CHUNK;
        t.part_chunks[bp + k] = make_int4(s, b, min(b + CHUNK, G.slot_off + G.nslot), 0);
    }
    for(int k = 0; k < nc; ++k)
    {
        const int b = G.cell_off + k * CHUNK;
        t.cell_chunks[bc + k] = make_int4(s, b, min(b + CHUNK, G.cell_off + G.ncell), 0);
    }
}

__global__ void __launch_bounds__(TPB) k_cells_zero(TermArrays t)
{
    const int n = t.work[1];
    for(int c = blockIdx.x; c < n; c += gridDim.x)
    {
        const int4 w = t.cell_chunks[c];
        const int cell = w.y + threadIdx.x;
        if(cell < w.z) {t.cell_count[cell] = 0; t.cell_fill[cell] = 0;}
    }
}

__global__ void __launch_bounds__(TPB) k_cells_assign(Arena a, int g, TermArrays t)
{
    const int n = t.work[0];
    for(int c = blockIdx.x; c < n; c += gridDim.x)
    {
        const int4 w = t.part_chunks[c];
        const int p = w.y + threadIdx.x;      // participant index (same range as slots)
        if(p >= w.z) {continue;}
        const GlobalParams& G = a.sys[w.x].g[g];
        const double4 r = a.pos[t.part_particle[p]];
        const int cx = cell_coord(r.x, G, 0);
        const int cy = cell_coord(r.y, G, 1);
        const int cz = cell_coord(r.z, G, 2);
        const int cell = G.cell_off + cx + G.dims[0] * (cy + G.dims[1] * cz);
        t.part_cell[p] = cell;
        atomicAdd(&t.cell_count[cell], 1);
    }
}

// exclusive scan of one flagged system's cells per block (SCAN_ITEMS cells
// per thread and pass); cell_start of the system's first cell is its first
// slot
constexpr int SCAN_ITEMS = 4;
__global__ void __launch_bounds__(SCAN_TPB) k_scan_sys(Arena a, int g, TermArrays t)
{
    const int nf = t.work[2];
    __shared__ int warp_tot[SCAN_TPB / 32];
    __shared__ int carry;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for(int f = blockIdx.x; f < nf; f += gridDim.x)
    {
        const GlobalParams& G = a.sys[t.flagged[f]].g[g];
        if(threadIdx.x == 0) {carry = G.slot_off;}
        __syncthreads();
        for(int base = 0; base < G.ncell; base += SCAN_TPB * SCAN_ITEMS)
        {
            const int first = base + threadIdx.x * SCAN_ITEMS;     // this thread's cells
            int v[SCAN_ITEMS];
            int sum = 0;
#pragma unroll
            for(int q = 0; q < SCAN_ITEMS; ++q)
            {
                v[q] = first + q < G.ncell ? t.cell_count[G.cell_off + first + q] : 0;
                sum += v[q];
            }
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
            int run = carry + warp_tot[w] + incl - sum;
#pragma unroll
            for(int q = 0; q < SCAN_ITEMS; ++q)
            {
                if(first + q < G.ncell) {t.cell_start[G.cell_off + first + q] = run;}
                run += v[q];
            }
            __syncthreads();
            if(threadIdx.x == SCAN_TPB - 1) {carry = run;}
            __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(TPB) k_cells_scatter(TermArrays t, int* slot_tmp)
{
    const int n = t.work[0];
    for(int c = blockIdx.x; c < n; c += gridDim.x)
    {
        const int4 w = t.part_chunks[c];
        const int p = w.y + threadIdx.x;
        if(p >= w.z) {continue;}
        const int cell = t.part_cell[p];
        const int k = atomicAdd(&t.cell_fill[cell], 1);
        slot_tmp[t.cell_start[cell] + k] = p;
    }
}

// rank sort of each cell's members by participant index, so that the slot
// order depends only on the cell assignment.  A warp takes 32 cells: each
// lane sorts a small cell (up to SMALL members) by itself, then the warp sorts
// the larger ones together, one after the other.
constexpr int SMALL = 8;
__global__ void __launch_bounds__(TPB) k_cells_sort(TermArrays t, const int* slot_tmp)
{
    const int n = t.work[1];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned full = 0xffffffffu;
    for(int c = blockIdx.x; c < n; c += gridDim.x)
    {
        const int4 w = t.cell_chunks[c];
        for(int cb = w.y + wid * 32; cb < w.z; cb += TPB)
        {
            const int cell = cb + lane;
            int b = 0, m = 0;
            if(cell < w.z) {b = t.cell_start[cell]; m = t.cell_count[cell];}
            if(m <= SMALL)
            {
                for(int e = 0; e < m; ++e)
                {
                    const int v = slot_tmp[b + e];
                    int rank = 0;
                    for(int u = 0; u < m; ++u) {rank += slot_tmp[b + u] < v ? 1 : 0;}
                    t.slot_part[b + rank] = v;
                }
            }
            unsigned big = __ballot_sync(full, m > SMALL);
            while(big)
            {
                const int src = __ffs(big) - 1;
                big &= big - 1;
                const int bb = __shfl_sync(full, b, src), mm = __shfl_sync(full, m, src);
                for(int e = lane; e < mm; e += 32)
                {
                    const int v = slot_tmp[bb + e];
                    int rank = 0;
                    for(int u = 0; u < mm; ++u) {rank += slot_tmp[bb + u] < v ? 1 : 0;}
                    t.slot_part[bb + rank] = v;
                }
            }
        }
    }
}

__global__ void __launch_bounds__(TPB) k_slots_setup(Arena a, TermArrays t)
{
    const int n = t.work[0];
    for(int c = blockIdx.x; c < n; c += gridDim.x)
    {
        const int4 w = t.part_chunks[c];
        const int s = w.y + threadIdx.x;
        if(s >= w.z) {continue;}
        const int p = t.slot_part[s];
        const int i = t.part_particle[p];
        const double4 r = a.pos[i];
        t.slot_particle[s] = i;
        t.slot_of[i]       = s;
        t.slot_lead[s]     = t.part_lead[p];
        t.slot_sys[s]      = w.x;
        t.slot_pd[s]       = make_double4(r.x, r.y, r.z, t.part_p0[p]);
        if(t.part_p1) {t.slot_p1[s] = t.part_p1[p];}
    }
}

// A slot's exclusion row staged in shared memory once per slot: the CSR row of
// particle i holds every particle excluded together with i (the relation is
// symmetric: topology distance and molecule rules; i itself included), so
// is_excluded(min(i, j), max(i, j)) is "j is in i's row" -- a comparison
// against the staged row instead of a chain of dependent loads per candidate.
// Rows longer than EXMAX are scanned in global memory as before.
constexpr int EXMAX = 16;
struct ExRow {
    int n;              // entries staged, or -1: the row is longer than EXMAX
    int mol;            // molecule of particle i
    int v[EXMAX];       // sorted excluded partners of i
};
// lanes [0, nl) of the slot's group stage particle i's row (every lane of the
// group must call it, then synchronise the group before reading the row)
__device__ __forceinline__ void stage_ex_row(const Arena& a, int g, int i, int gl, int nl, ExRow& r)
{
    const long long b = a.ex_start[g][i], e = a.ex_start[g][i + 1];
    const int n = (int)(e - b);
    if(gl == 0) {r.n = n <= EXMAX ? n : -1; r.mol = a.mol[i];}
    if(n <= EXMAX) {for(int k = gl; k < n; k += nl) {r.v[k] = a.ex_idx[g][b + k];}}
}
__device__ __forceinline__ bool is_excluded(const Arena& a, int g, int ignore_mol, int i, int j);
// is_excluded(min(i, j), max(i, j)) for the slot's particle i and candidate j
__device__ __forceinline__ bool excluded_staged(const Arena& a, int g, int ignore_mol, const ExRow& r, int i, int j)
{
    if(ignore_mol != IGN_NOTHING)
    {
        const int mj = a.mol[j];
        if(ignore_mol == IGN_SELF   && r.mol == mj) {return true;}
        if(ignore_mol == IGN_OTHERS && r.mol != mj) {return true;}
    }
    if(r.n < 0) {return is_excluded(a, g, IGN_NOTHING, i < j ? i : j, i < j ? j : i);}
    for(int k = 0; k < r.n; ++k)
    {
        const int x = r.v[k];
        if(x > j) {break;}
        if(x == j) {return true;}
    }
    return false;
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

// Half lists keep a pair in the list of its lower slot only: a stencil cell's
// slot range [start, start + count) is cut to the slots above s (slots are in
// cell order, so a cell is one range), which leaves the full list's words
// above s in their order.  The full lists are symmetric (the distance test,
// the leading-participant rule and the exclusions do not depend on which
// partner asks), so every pair of them is in exactly one half list.
__device__ __forceinline__ void clip_half(int& start, int& count, int s)
{
    const int lo = max(start, s + 1);
    count = max(0, start + count - lo);
    start = lo;
}

// One warp per slot.  The 27 stencil cells (in the reference's order: z, y, x
// from -1 to +1) are flattened into one candidate sequence that the 32 lanes
// walk together; the distance test reads the cell-ordered slot coordinates
// (consecutive candidates are consecutive in memory), the topology checks run
// only for candidates inside the list radius, and an ordered ballot
// compaction keeps the output order identical to a serial walk.
__global__ void __launch_bounds__(TPB) k_build_list(Arena a, int g, TermArrays t)
{
    const int n = t.work[0];
    const int cap = t.cap;
    const long long np = t.np;
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    // every warp of the grid takes the next (chunk, slot) pair, so that all
    // warps have work even when only a few systems rebuild
    __shared__ ExRow ex_rows[TPB / 32];
    ExRow& exr = ex_rows[threadIdx.x >> 5];
    const long long nwork = (long long)n * CHUNK;
    const long long wstride = (long long)gridDim.x * (TPB / 32);
    for(long long gw = (long long)blockIdx.x * (TPB / 32) + (threadIdx.x >> 5); gw < nwork; gw += wstride)
    {
        const int4 w = t.part_chunks[gw / CHUNK];
        const int s = w.y + (int)(gw % CHUNK);
        if(s >= w.z) {continue;}
        const int sys = w.x;
        const SysDev& S = a.sys[sys];
        const GlobalParams& G = S.g[g];
        const bool periodic = S.boundary == B_PERIODIC;
        const int dx_ = G.dims[0], dy_ = G.dims[1], dz_ = G.dims[2];
        const bool wrap = periodic || G.hashed;
        const double rl2 = G.rl2;
        {
            const int i = t.slot_particle[s];
            const bool lead_i = t.slot_lead[s] != 0;
            const double4 ri = t.slot_pd[s];
            __syncwarp();                        // the previous slot's row is no longer read
            stage_ex_row(a, g, i, lane, 32, exr);
            __syncwarp();
            const int cx = cell_coord(ri.x, G, 0);
            const int cy = cell_coord(ri.y, G, 1);
            const int cz = cell_coord(ri.z, G, 2);
            // this lane's stencil cell
            int cstart = 0, ccount = 0;
            if(lane < 27)
            {
                int x = cx + lane % 3 - 1, y = cy + (lane / 3) % 3 - 1, z = cz + lane / 9 - 1;
                bool inside = true;
                if(wrap)
                {
                    x = x < 0 ? x + dx_ : (x >= dx_ ? x - dx_ : x);
                    y = y < 0 ? y + dy_ : (y >= dy_ ? y - dy_ : y);
                    z = z < 0 ? z + dz_ : (z >= dz_ ? z - dz_ : z);
                }
                else if(x < 0 || y < 0 || z < 0 || x >= dx_ || y >= dy_ || z >= dz_) {inside = false;}
                if(inside)
                {
                    const int cell = G.cell_off + x + dx_ * (y + dy_ * z);
                    cstart = t.cell_start[cell];
                    ccount = t.cell_count[cell];
                    if(t.half) {clip_half(cstart, ccount, s);}
                }
            }
            int incl = ccount;
#pragma unroll
            for(int o = 1; o < 32; o <<= 1)
            {
                const int y = __shfl_up_sync(full, incl, o);
                if(lane >= o) {incl += y;}
            }
            const int excl = incl - ccount;
            const int total = __shfl_sync(full, incl, 31);
            int count = 0;
            for(int base = 0; base < total; base += 32)
            {
                const int k = base + lane;
                // cell of candidate k: the last stencil lane whose range starts at or before k
                int L = 0;
#pragma unroll
                for(int b = 16; b > 0; b >>= 1)
                {
                    const int cand = L + b;
                    const int e = __shfl_sync(full, excl, cand < 32 ? cand : 31);
                    if(cand < 27 && e <= k) {L = cand;}
                }
                const int q = __shfl_sync(full, cstart, L) + (k - __shfl_sync(full, excl, L));
                bool keep = false;
                if(k < total && q != s)
                {
                    const double4 rj = t.slot_pd[q];
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
                    if(l2 < rl2)
                    {
                        const int j = t.slot_particle[q];
                        const bool lead_lo = (i < j) ? lead_i : (t.slot_lead[q] != 0);
                        keep = lead_lo && !excluded_staged(a, g, G.ignore_mol, exr, i, j);
                    }
                }
                const unsigned m = __ballot_sync(full, keep);
                if(keep)
                {
                    const int pos = count + __popc(m & ((1u << lane) - 1u));
                    if(pos < cap) {t.nbr[nbr_pos(pos, s, np, t.tpp, cap, t.slot_major)] = q;}
                }
                count += __popc(m);
            }
            if(lane == 0)
            {
                t.nnb[s] = count < cap ? count : cap;
                atomicMax(t.max_count, count);
                if(count > cap) {atomicOr(&a.sys[sys].status, ST_LIST_OVERFLOW);}
            }
        }
    }
}

// The same list build with LPS lanes per slot (4, 8 or 16): a warp builds 32 /
// LPS lists at once, so that short candidate sequences (a few partners per
// stencil) do not leave most of a warp idle while it waits on memory.  A
// group's 27 stencil ranges go through shared memory; candidate k of the
// flattened sequence belongs to the last stencil cell whose range starts at
// or before k; the ordered compaction within the group keeps the serial
// walk's output order, so the lists are the same word for word.
template<int LPS>
__global__ void __launch_bounds__(TPB) k_build_list_sub(Arena a, int g, TermArrays t)
{
    constexpr int GROUPS = TPB / LPS;              // slot groups per block
    constexpr int WG = 32 / LPS;                   // slot groups per warp
    constexpr int CPL = (27 + LPS - 1) / LPS;      // stencil cells per lane
    __shared__ int c_start[GROUPS][27];
    __shared__ int c_excl[GROUPS][28];             // exclusive prefix; [27] = total
    __shared__ ExRow ex_rows[GROUPS];
    const int n = t.work[0];
    const int cap = t.cap;
    const long long np = t.np;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int grp = threadIdx.x / LPS, gl = threadIdx.x % LPS;
    const unsigned full = 0xffffffffu;
    const unsigned gmask = ((LPS == 32) ? full : ((1u << LPS) - 1u)) << (lane - gl);
    const long long nwork = (long long)n * CHUNK;
    const long long stride = (long long)gridDim.x * GROUPS;
    // warp-uniform loop over rounds; group (lane / LPS) of the warp takes item base + lane / LPS
    for(long long base = (long long)blockIdx.x * GROUPS + warp * WG; base < nwork; base += stride)
    {
        const long long item = base + lane / LPS;
        bool valid = item < nwork;
        int s = 0, sys = 0;
        if(valid)
        {
            const int4 w = t.part_chunks[item / CHUNK];
            s = w.y + (int)(item % CHUNK);
            sys = w.x;
            valid = s < w.z;
        }
        const SysDev& S = a.sys[sys];
        const GlobalParams& G = S.g[g];
        const bool periodic = S.boundary == B_PERIODIC;
        const int dx_ = G.dims[0], dy_ = G.dims[1], dz_ = G.dims[2];
        const bool wrap = periodic || G.hashed;
        const double rl2 = G.rl2;
        int i = 0;
        bool lead_i = false;
        double4 ri = make_double4(0.0, 0.0, 0.0, 0.0);
        if(valid)
        {
            i = t.slot_particle[s];
            lead_i = t.slot_lead[s] != 0;
            ri = t.slot_pd[s];
            stage_ex_row(a, g, i, gl, LPS, ex_rows[grp]);
            const int cx = cell_coord(ri.x, G, 0);
            const int cy = cell_coord(ri.y, G, 1);
            const int cz = cell_coord(ri.z, G, 2);
            for(int k = gl * CPL; k < gl * CPL + CPL && k < 27; ++k)   // this lane's block of stencil cells
            {
                int x = cx + k % 3 - 1, y = cy + (k / 3) % 3 - 1, z = cz + k / 9 - 1;
                bool inside = true;
                if(wrap)
                {
                    x = x < 0 ? x + dx_ : (x >= dx_ ? x - dx_ : x);
                    y = y < 0 ? y + dy_ : (y >= dy_ ? y - dy_ : y);
                    z = z < 0 ? z + dz_ : (z >= dz_ ? z - dz_ : z);
                }
                else if(x < 0 || y < 0 || z < 0 || x >= dx_ || y >= dy_ || z >= dz_) {inside = false;}
                int cs = 0, cc = 0;
                if(inside)
                {
                    const int cell = G.cell_off + x + dx_ * (y + dy_ * z);
                    cs = t.cell_start[cell];
                    cc = t.cell_count[cell];
                    if(t.half) {clip_half(cs, cc, s);}
                }
                c_start[grp][k] = cs;
                c_excl[grp][k] = cc;
            }
        }
        __syncwarp();
        // exclusive prefix of the 27 counts: within each lane's block, then
        // across the group's lanes with shuffles
        {
            int cnt[CPL];
            int sum = 0;
#pragma unroll
            for(int j = 0; j < CPL; ++j)
            {
                const int k = gl * CPL + j;
                cnt[j] = (valid && k < 27) ? c_excl[grp][k] : 0;
                sum += cnt[j];
            }
            int incl = sum;
#pragma unroll
            for(int o = 1; o < LPS; o <<= 1)
            {
                const int y = __shfl_up_sync(full, incl, o, LPS);
                if(gl >= o) {incl += y;}
            }
            int run = incl - sum;
#pragma unroll
            for(int j = 0; j < CPL; ++j)
            {
                const int k = gl * CPL + j;
                if(valid && k < 27) {c_excl[grp][k] = run;}
                run += cnt[j];
            }
            if(valid && gl == LPS - 1) {c_excl[grp][27] = incl;}
        }
        __syncwarp();
        const int total = valid ? c_excl[grp][27] : 0;
        int tmax = total;
#pragma unroll
        for(int o = LPS; o < 32; o <<= 1) {tmax = max(tmax, __shfl_xor_sync(full, tmax, o));}
        int count = 0;
        int lo = 0;         // the last stencil cell whose range starts at or before k: k only grows, so
                            // the lane walks forward from its previous cell
        for(int b = 0; b < tmax; b += LPS)
        {
            const int k = b + gl;
            bool keep = false;
            int q = 0;
            if(k < total)
            {
                while(lo < 26 && c_excl[grp][lo + 1] <= k) {++lo;}
                q = c_start[grp][lo] + (k - c_excl[grp][lo]);
                if(q != s)
                {
                    const double4 rj = t.slot_pd[q];
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
                    if(l2 < rl2)
                    {
                        const int j = t.slot_particle[q];
                        const bool lead_lo = (i < j) ? lead_i : (t.slot_lead[q] != 0);
                        keep = lead_lo && !excluded_staged(a, g, G.ignore_mol, ex_rows[grp], i, j);
                    }
                }
            }
            const unsigned m = __ballot_sync(full, keep) & gmask;
            if(keep)
            {
                const int pos = count + __popc(m & ((1u << lane) - 1u));
                if(pos < cap) {t.nbr[nbr_pos(pos, s, np, t.tpp, cap, t.slot_major)] = q;}
            }
            count += __popc(m);
        }
        if(valid && gl == 0)
        {
            t.nnb[s] = count < cap ? count : cap;
            atomicMax(t.max_count, count);
            if(count > cap) {atomicOr(&a.sys[sys].status, ST_LIST_OVERFLOW);}
        }
        __syncwarp();
    }
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
    if(s == 0) {t.work[0] = 0; t.work[1] = 0; t.work[2] = 0; *t.any_rebuild = 0;}
}

__global__ void k_scatter_param(TermArrays t, double* w)
{
    const long long p = (long long)blockIdx.x * TPB + threadIdx.x;
    if(p < t.np) {w[t.part_particle[p]] = t.part_p0[p];}
}

inline unsigned blocks(long long n, int tpb = TPB) {return (unsigned)((n + tpb - 1) / tpb);}

}  // namespace

void launch_scatter_param(const TermArrays& t, double* w, cudaStream_t s)
{
    if(!t.on || t.np == 0) {return;}
    k_scatter_param<<<blocks(t.np), TPB, 0, s>>>(t, w);
    note_launches(1);
}

void launch_rebuild(const Arena& a, int g, TermArrays& t, int force_all, cudaStream_t s)
{
    if(!t.on || t.np == 0) {return;}
    k_plan        <<<blocks(a.nsys, 128), 128, 0, s>>>(a, g, t, force_all);
    k_cells_zero  <<<GRID, TPB, 0, s>>>(t);
    k_cells_assign<<<GRID, TPB, 0, s>>>(a, g, t);
    k_scan_sys    <<<min(a.nsys, 1024), SCAN_TPB, 0, s>>>(a, g, t);
    k_cells_scatter<<<GRID, TPB, 0, s>>>(t, t.slot_particle);
    k_cells_sort  <<<GRID, TPB, 0, s>>>(t, t.slot_particle);
    k_slots_setup <<<GRID, TPB, 0, s>>>(a, t);
    if(t.build_lanes == 4)       {k_build_list_sub<4> <<<GRID, TPB, 0, s>>>(a, g, t);}
    else if(t.build_lanes == 8)  {k_build_list_sub<8> <<<GRID, TPB, 0, s>>>(a, g, t);}
    else if(t.build_lanes == 16) {k_build_list_sub<16><<<GRID, TPB, 0, s>>>(a, g, t);}
    else                         {k_build_list        <<<GRID, TPB, 0, s>>>(a, g, t);}
    k_rebuild_done<<<blocks(a.nsys, 128), 128, 0, s>>>(a, g, t, force_all);
    note_launches(9);
}

}  // namespace mjg
