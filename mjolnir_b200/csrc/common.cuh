// Shared device-side definitions of the B200 Mjolnir hot path.
//
// Layout in HBM (one "arena" packs every resident system back to back):
//   pos, vel        double4 per particle (w unused)       -- FP64 master state
//   force           32 B per particle: double4 (FP64 mode) or longlong4 of
//                   fixed-point values (mixed mode, 2^-FX_SHIFT resolution)
//   coef            double4 per particle: {halfdt/m, exp(-gamma dt), noise, halfdt | dt}
//   psys            int32 per particle: system slot
// Per global term (ExcludedVolume, DebyeHuckel, LennardJones) the participants
// are renumbered into "slots" in cell order at every list rebuild; the
// neighbour list is stored column-major: nbr[k * nslots + s] = slot of the k-th
// partner of slot s, so that a warp of consecutive slots reads coalesced.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mjg {

enum Term : int { T_BOND = 0, T_ANGLE = 1, T_DIHEDRAL = 2, T_EXV = 3, T_DH = 4, T_LJ = 5, NTERMS = 6 };
enum { G_EXV = 0, G_DH = 1, G_LJ = 2, NGLOBAL = 3 };
enum Boundary : int { B_UNLIMITED = 0, B_PERIODIC = 1 };
enum Integrator : int { I_BAOAB = 0, I_VV = 1, I_UNDERDAMPED = 2, I_GJF = 3, I_GBAOAB = 4 };
enum IgnoreMol : int { IGN_NOTHING = 0, IGN_SELF = 1, IGN_OTHERS = 2 };
enum Precision : int { P_FP64 = 0, P_MIXED = 1 };

// status bits written by kernels into SysDev::status (never a trap)
enum : int {
    ST_LIST_OVERFLOW  = 1,   // a neighbour list exceeded its capacity
    ST_FIXED_OVERFLOW = 2,   // a force left the fixed-point range
    ST_NONFINITE      = 4,   // a non-finite force or position
};

// Fixed-point forces: value = integer * 2^-FX_SHIFT.  Conversion uses the
// 1.5 * 2^52 rounding constant so that it runs on the FP64 pipe; it is exact
// round-to-nearest for |value| * 2^FX_SHIFT < 2^50.
constexpr int    FX_SHIFT     = 28;
constexpr double FX_SCALE     = 268435456.0;            // 2^28
constexpr double FX_INV_SCALE = 1.0 / 268435456.0;
constexpr double FX_LIMIT     = 1125899906842624.0;     // 2^50
constexpr double FX_MAGIC     = 6755399441055744.0;     // 1.5 * 2^52

// potential of the third global term: LennardJones (its own interaction,
// forcefield/global/GlobalPairLennardJonesInteraction.hpp) or a potential of
// the family through the generic pair loop (GlobalPairInteraction.hpp:148-213)
enum LjKind { LJ_PLAIN = 0, LJ_WCA = 1, LJ_ATTRACTIVE = 2, LJ_UNIFORM = 3 };
// potential of the first global term: ExcludedVolume (its own interaction,
// GlobalPairExcludedVolumeInteraction.hpp) or InversePower /
// HardCoreExcludedVolume through the generic pair loop
enum ExvKind { EXV_PLAIN = 0, EXV_INVERSE_POWER = 1, EXV_HARD_CORE = 2 };
constexpr double SIXTH_ROOT_OF_TWO = 1.12246204831;   // WCAPotential.hpp default_cutoff

struct GlobalParams {       // per system, per global term
    double cutoff;          // max_cutoff_length
    double margin;          // relative skin
    double current_margin;  // remaining skin (reduce_margin bookkeeping)
    double rl2;             // (cutoff (1 + margin))^2, list radius squared
    // potential constants
    double eps;             // EXV epsilon
    double cutoff_ratio;
    double cutoff_ratio_sq;
    double coef_at_cutoff;
    double debye, inv_debye, abs_cutoff, inv4pi;   // DH
    // cell grid
    double origin[3];
    double inv_w[3];        // reciprocal cell width
    int    dims[3];
    int    hashed;          // unlimited boundary: cell coordinates wrap modulo dims
    int    cell_off;        // first global cell of this system
    int    ncell;
    int    slot_off;        // first slot of this system (participant offset)
    int    nslot;
    int    ignore_mol;      // IgnoreMol
    int    rebuild;         // set by the margin kernel, cleared after a rebuild
    int    rebuilds;        // rebuild counter
    int    kind;            // the term's potential (ExvKind for the first, LjKind for the third)
    int    power;           // InversePower exponent n
    int    on;
};

struct SysDev {
    long long off, n;       // particle range in the arena
    int    boundary, integrator;
    double lower[3], upper[3], width[3], halfw[3];
    unsigned long long seed;
    unsigned long long step;
    unsigned long long max_disp2;   // bits of a non-negative double (atomicMax)
    int    status;
    int    frozen;          // 1: the system does not advance (set by the host between chunks)
    int    uniform_coef;    // 1: every particle has the integrator coefficients `coef` (the per-particle
                            // array is then not read)
    double4 coef;
    double energy[NTERMS];
    GlobalParams g[NGLOBAL];
};

// ---------------------------------------------------------------- helpers

__device__ __forceinline__ long long fx_from_double(double v)
{
    // round(v * 2^FX_SHIFT) without a D2I conversion
    const double s = v * FX_SCALE + FX_MAGIC;
    return __double_as_longlong(s) - __double_as_longlong(FX_MAGIC);
}
__device__ __forceinline__ double fx_to_double(long long v)
{
    return (double)v * FX_INV_SCALE;
}

// Minimum image of core/BoundaryCondition.hpp:81-91 with the reference's
// branch order; explicit _rn ops keep it free of contractions.
__device__ __forceinline__ double min_image(double d, double halfw, double width)
{
    if(d < -halfw)       {d = __dadd_rn(d, width);}
    else if(d >= halfw)  {d = __dsub_rn(d, width);}
    return d;
}

// ------------------------------------------------------- Philox4x32-10
// Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11: 10 rounds of the 4x32 Philox S-box with Weyl key schedule.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
#pragma unroll
    for(int r = 0; r < 10; ++r)
    {
        if(r) {k.x += 0x9E3779B9u; k.y += 0xBB67AE85u;}
        const unsigned hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const unsigned hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    }
    return c;
}

// Three N(0,1) deviates for (system seed, particle, step) by Box-Muller.
__device__ __forceinline__ void gaussian3(unsigned long long seed, unsigned long long particle,
                                          unsigned long long step, double& g0, double& g1, double& g2)
{
    const uint4 x = philox4x32_10(
        make_uint4((unsigned)particle, (unsigned)(particle >> 32), (unsigned)step, (unsigned)(step >> 32)),
        make_uint2((unsigned)seed, (unsigned)(seed >> 32)));
    const double two32 = 2.3283064365386963e-10;   // 2^-32
    const double u0 = ((double)x.x + 0.5) * two32;
    const double u1 = (double)x.y * two32;
    const double u2 = ((double)x.z + 0.5) * two32;
    const double u3 = (double)x.w * two32;
    const double r0 = sqrt(-2.0 * log(u0));
    const double r1 = sqrt(-2.0 * log(u2));
    double s1, c1, s3, c3;
    sincospi(2.0 * u1, &s1, &c1);
    sincospi(2.0 * u3, &s3, &c3);
    g0 = r0 * c1;
    g1 = r0 * s1;
    g2 = r1 * c3;
}

// Blocked column-major list layout: partner k of slot s.  With tpp threads per
// slot, the tpp lanes of a group read tpp consecutive words, and consecutive
// groups read consecutive blocks; tpp = 1 is plain column-major.
__host__ __device__ __forceinline__ long long nbr_index(long long k, long long s, long long np, int tpp)
{
    return ((k / tpp) * np + s) * tpp + (k % tpp);
}
// Slot-major layout (dense terms): each slot's list contiguous, `cap` words
// per slot, so that one bulk copy engine request brings a whole list to L2.
__host__ __device__ __forceinline__ long long nbr_pos(long long k, long long s, long long np, int tpp, int cap,
                                                      int slot_major)
{
    return slot_major ? s * cap + k : nbr_index(k, s, np, tpp);
}

// Cell coordinate of x along one axis (PeriodicGridCellList::calc_index for a
// periodic system; a wrapped hash of the unbounded grid otherwise).
__device__ __forceinline__ int cell_coord(double x, const GlobalParams& g, int axis)
{
    const double t = floor(__dmul_rn(__dsub_rn(x, g.origin[axis]), g.inv_w[axis]));
    const int d = g.dims[axis];
    if(g.hashed)
    {
        long long c = (long long)t % d;
        if(c < 0) {c += d;}
        return (int)c;
    }
    long long c = (long long)t;
    if(c < 0) {c = 0;}
    if(c > d - 1) {c = d - 1;}
    return (int)c;
}

}  // namespace mjg
