// Host-side launch wrappers of every kernel of the hot path.  All launches go
// to the stream given; nothing here allocates or synchronises.
#pragma once
#include "common.cuh"

namespace mjg {

// Device-resident arrays of one arena (all pointers are device pointers).
struct Arena {
    int       precision;        // Precision
    long long n;                // particles
    int       nsys;
    int       any_frozen;       // some system is frozen (kernels read the per-system flag only then)
    SysDev*   sys;              // [nsys]
    double4*  pos;
    double4*  vel;
    void*     force;            // double4 (P_FP64) or longlong4 (P_MIXED)
    double4*  coef;             // BAOAB {halfdt/m, e^-g dt, noise, halfdt}; VV {halfdt/m, 1, 0, dt};
                                // UnderdampedLangevin {1/m, gamma, noise sigma, dt};
                                // G-JF {halfdt/m, a, beta, dt}
    double4*  accel;            // UnderdampedLangevin: acceleration with noise; G-JF: {1/2m, b/m, b dt}
                                // (nullptr: no system of either kind)
    int*      psys;
    double*   staging;          // [3 n] host-layout staging for copies
    // exclusions (per global term): excluded partners of every particle,
    // sorted, CSR over particles
    const long long* ex_start[NGLOBAL];
    const int*       ex_idx[NGLOBAL];
    const int*       mol;       // molecule id per particle (global numbering)
    // slot coordinates of every global term, written by the integrator
    // through the particle -> slot map (nullptr: term off)
    double4*         slot_pd[NGLOBAL];
    const int*       slot_of[NGLOBAL];
    const double*    slot_w[NGLOBAL];   // [n] the term's parameter of each particle (slot_pd.w)
};

// Per global term arrays (participants grouped by system, input order inside).
struct TermArrays {
    int        on;
    long long  np;              // participants (= slots)
    int        ncell;           // total cells over all systems
    int        cap;             // neighbour capacity per slot (a multiple of tpp)
    int        tpp;             // threads per slot of the pair kernel (1, 2, 4, 8, 16, 32)
    int        unroll;          // partners requested per batch by the force launch (1, 2, 4)
    int        schedule;        // force launch: 0 = slot per tpp threads, 1 = warp-balanced (mixed),
                                // 2 = one thread per slot reading tpp-word blocks of its list,
                                // 3 = as 2 with a block's threads ordered by list length,
                                // 4 = as 0 with a block's thread groups ordered by list length,
                                // 5 = as 0 on the slot-major layout, each group's list brought
                                //     to L2 by one bulk prefetch when the group starts
    int        any_periodic;    // some system with this term has a periodic box
    int        build_lanes;     // lanes per slot of the list build (8, 16 or 32)
    int        slot_major;      // list layout: 0 blocked by tpp (nbr_index), 1 slot-major (nbr_pos)
    int        half;            // list form: 0 full (a pair in both partners' lists), 1 half (mixed
                                // form only: a pair in the list of its lower slot alone, and the
                                // force launch adds the negated pair force to the partner)
    int        fe_energy;       // energy-only launch: sum the energy as calc_force_and_energy does
                                // (the generic pair loop skips pairs whose force is zero,
                                // GlobalPairInteraction.hpp:148-213) instead of calc_energy's
                                // every listed pair
    const int* part_particle;   // [np] global particle index
    const double* part_p0;      // [np] radius / charge / sigma
    const double* part_p1;      // [np] LJ epsilon
    const unsigned char* part_lead; // [np] leading participant
    const int* part_sys;        // [np]
    int*       part_cell;       // [np]
    int*       cell_count;      // [ncell]
    int*       cell_start;      // [ncell + 1]
    int*       cell_fill;       // [ncell]
    int*       work;            // [3] rebuild work counters
    int4*      part_chunks;     // rebuild work: participant chunks {sys, begin, end}
    int4*      cell_chunks;     // rebuild work: cell chunks
    int*       flagged;         // [nsys] systems rebuilding this step
    int*       slot_part;       // [np] participant of slot (cell order)
    int*       slot_particle;   // [np] global particle of slot
    unsigned char* slot_lead;   // [np]
    int*       slot_sys;        // [np]
    double4*   slot_pd;         // [np] x, y, z, p0 (kept current by the integrator)
    int*       slot_of;         // [n] slot of each particle of the arena, -1 if none
    double*    slot_p1;         // [np] LJ epsilon per slot
    int*       nnb;             // [np] partners per slot
    int*       nbr;             // [cap * np] column-major
    int*       max_count;       // [1] largest list seen at the last build
    int*       any_rebuild;     // [1]
};

void launch_unpack_state(const Arena& a, const double* src_pos, const double* src_vel,
                         long long first, long long count, cudaStream_t s);
void launch_pack_state(const Arena& a, double* dst, int what, long long first, long long count,
                       cudaStream_t s);

// kick: apply the previous step's closing half-kick in the same pass
void launch_integrate_first(const Arena& a, cudaStream_t s, bool kick = false);
// UnderdampedLangevin: acceleration from the current forces and noise for the
// particles [first, first + count) (Integrator::initialize)
void launch_init_accel(const Arena& a, long long first, long long count, cudaStream_t s);
// accel[first + k] = src[3k .. 3k + 2] (host-layout staging)
void launch_set_accel(const Arena& a, const double* src, long long first, long long count, cudaStream_t s);
// Graph-conditional rebuilds: in a captured step each global term's rebuild
// sits in the body of an `if` node whose handle the margin kernel sets when
// some system flags that term; a step in which no system of the term needs
// new lists skips the rebuild's launches (on[g] = 0: no such node, the
// rebuild always runs and filters the flagged systems itself).
struct RebuildGate {
    int on[NGLOBAL];
    cudaGraphConditionalHandle handle[NGLOBAL];
};
void launch_margin(const Arena& a, TermArrays* t, cudaStream_t s, const RebuildGate& gate);
void launch_integrate_last(const Arena& a, cudaStream_t s);
void launch_zero_force(const Arena& a, cudaStream_t s);

void launch_rebuild(const Arena& a, int gterm, TermArrays& t, int force_all, cudaStream_t s);
// w[particle] = the term's parameter of each participant (radius, charge, sigma)
void launch_scatter_param(const TermArrays& t, double* w, cudaStream_t s);
// slot coordinates of a term's participants (before its force launch)
void launch_gather(const Arena& a, TermArrays& t, cudaStream_t s);
// gather: refresh the slot coordinates first (the step's launches rely on
// the integrator and the rebuild having done so)
void launch_pair(const Arena& a, int gterm, TermArrays& t, bool need_force, bool need_energy,
                 int calc_energy_form, cudaStream_t s, bool gather = true);

struct LocalArrays {
    long long nbond, nangle, ndihd;
    const int* bond_idx;   const double* bond_k;  const double* bond_v0;  const int* bond_sys;
    const int* angle_idx;  const double* angle_k; const double* angle_v0; const int* angle_sys;
    const int* dihd_idx;   const double* dihd_k;  const int* dihd_n; const double* dihd_v0;
    const int* dihd_sys;
    // float parameters of the mixed form: {k, v0}, {k, v0}, {k, cos(n v0), sin(n v0), n}
    const float2* bond_kv;
    const float2* angle_kv;
    const float4* dihd_p;
    // terms sorted by their smallest particle index; window w of 256 particles
    // owns terms win_x[w] .. win_x[w + 1]
    int nwin;
    const long long* win_bond;
    const long long* win_angle;
    const long long* win_dihd;
};
void launch_local(const Arena& a, const LocalArrays& l, int which_mask, bool need_force,
                  bool need_energy, int calc_energy_form, cudaStream_t s);

void launch_clear_energy(const Arena& a, cudaStream_t s);
void launch_count_cut(const Arena& a, int g, TermArrays& t, int sys, unsigned long long* out,
                      cudaStream_t s);
// reads `bytes` (a multiple of 16) at p, leaving clean lines in L2 (timing
// aid: evicts dirty lines after a flush write)
void launch_read_sweep(const void* p, size_t bytes, int* sink, cudaStream_t s);
// coef[first + k].z = noise[k] (the Langevin noise coefficient) for k < count
void launch_set_noise(const Arena& a, const double* noise, long long first, long long count,
                      cudaStream_t s);
// writes host-layout forces [3 count] (staging) into the arena's force array
void launch_set_force(const Arena& a, const double* src, long long first, long long count,
                      cudaStream_t s);

// kernel launch accounting (every wrapper reports what it enqueued)
void note_launches(int k);

}  // namespace mjg
