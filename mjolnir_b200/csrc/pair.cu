// Global pair forces and energies over the full Verlet lists.
//
//   ExcludedVolume  forcefield/global/GlobalPairExcludedVolumeInteraction.hpp:148-195
//   DebyeHuckel     forcefield/global/GlobalPairInteraction.hpp:148-213 with
//                   forcefield/global/DebyeHuckelPotential.hpp:44-61
//   LennardJones    forcefield/global/GlobalPairLennardJonesInteraction.hpp:148-198
//                   with the Lorentz-Berthelot rule (ParameterList.hpp:240-251)
//
// One thread owns one slot (particle) and walks its column-major list, so a
// warp of 32 consecutive slots -- 32 spatial neighbours after the cell-order
// renumbering -- loads 32 consecutive list words per step and mostly the same
// partner coordinates.  The owner accumulates and writes its particle's force
// once: no scattered atomics.  Each pair is evaluated from both sides (the
// reference evaluates it once and applies Newton's third law).
//
// P_FP64  : the reference's arithmetic in FP64 (the plain form).
// P_MIXED : the displacement and the cutoff test in FP64, the potential in FP32,
//           every pair force rounded to 2^-28 fixed point and summed as int64,
//           so the sum does not depend on list order or launch shape.
#include "kernels.cuh"

#include <type_traits>

namespace mjg {

namespace {

constexpr int TPB = 256;

__global__ void k_gather(Arena a, TermArrays t)
{
    const long long s = (long long)blockIdx.x * 256 + threadIdx.x;
    if(s >= t.np) {return;}
    const double4 r = a.pos[t.slot_particle[s]];
    double4& d = t.slot_pd[s];
    d.x = r.x; d.y = r.y; d.z = r.z;
}

template<int PREC>
struct Acc;

template<> struct Acc<P_FP64>
{
    double x = 0, y = 0, z = 0;
    __device__ __forceinline__ void add(double c, double dx, double dy, double dz, bool&)
    {
        x = fma(dx, c, x); y = fma(dy, c, y); z = fma(dz, c, z);
    }
    __device__ __forceinline__ void shfl_add(int o)
    {
        x += __shfl_xor_sync(0xffffffffu, x, o);
        y += __shfl_xor_sync(0xffffffffu, y, o);
        z += __shfl_xor_sync(0xffffffffu, z, o);
    }
    __device__ __forceinline__ void store(void* force, long long i) const
    {
        double4* f = static_cast<double4*>(force) + i;
        double4 v = *f;
        v.x += x; v.y += y; v.z += z;
        *f = v;
    }
};

template<> struct Acc<P_MIXED>
{
    long long x = 0, y = 0, z = 0;
    __device__ __forceinline__ void add(double c, double dx, double dy, double dz, bool& ovf)
    {
        const double fx = c * dx, fy = c * dy, fz = c * dz;
        const double m = fmax(fabs(fx), fmax(fabs(fy), fabs(fz)));
        ovf |= !(m < FX_LIMIT * FX_INV_SCALE);
        x += fx_from_double(fx); y += fx_from_double(fy); z += fx_from_double(fz);
    }
    // the mixed form's plain potentials: the FP32 pair coefficient c times
    // the FP64 displacement, each component rounded to the fixed-point grid
    // on the FP64 pipe (one conversion per pair instead of one per component
    // and coordinate); `bound` >= |c| |r| (|c| max(|r|^2, 1) or |c| |r|, in
    // FP32) flags a force outside the fixed-point range
    __device__ __forceinline__ void add_c(float c, float bound, double dx, double dy, double dz, bool& ovf)
    {
        const double cd = (double)c;
        ovf |= !(bound < (float)(FX_LIMIT * FX_INV_SCALE));
        x += fx_from_double(cd * dx);
        y += fx_from_double(cd * dy);
        z += fx_from_double(cd * dz);
    }
    __device__ __forceinline__ void shfl_add(int o)
    {
        x += __shfl_xor_sync(0xffffffffu, x, o);
        y += __shfl_xor_sync(0xffffffffu, y, o);
        z += __shfl_xor_sync(0xffffffffu, z, o);
    }
    // integer atomics: exact and order independent, so the force launches of
    // different terms and the bonded launch may run concurrently
    __device__ __forceinline__ void store(void* force, long long i) const
    {
        unsigned long long* f = reinterpret_cast<unsigned long long*>(static_cast<longlong4*>(force) + i);
        if(x) {atomicAdd(f + 0, (unsigned long long)x);}
        if(y) {atomicAdd(f + 1, (unsigned long long)y);}
        if(z) {atomicAdd(f + 2, (unsigned long long)z);}
    }
};

// Constants of one slot's pair evaluations and the evaluation of one pair
// (slot s, partner q).  PER: some system of the arena is periodic (the
// minimum image is applied where the system asks for it); without it the
// image code is compiled out.
template<int PREC, int G, bool NF, bool NE, bool PER, bool HALF = false>
struct PairEval {
    const SysDev* S;
    double4 pi;
    long long s;
    bool periodic;
    double crsq, coefc, eps, eps12, debye, inv_debye, abs_cut_sq, qi, inv4pi, epsi, cr;
    float eps12f, epsf, coefcf, debf, invdf, crsqf, wif;
    int kind, power;
    bool fe;                    // energy-only: the force-and-energy rule of the generic loop
    const double* slot_p1;
    void* force;
    const int* slot_particle;

    __device__ __forceinline__ PairEval(const Arena& a, const TermArrays& t, long long slot, int sys)
    {
        s = slot;
        S = &a.sys[sys];
        const GlobalParams& P = S->g[G];
        periodic = PER && S->boundary == B_PERIODIC;
        pi = t.slot_pd[slot];
        crsq  = P.cutoff_ratio_sq;
        cr    = P.cutoff_ratio;
        kind  = P.kind;
        power = P.power;
        coefc = P.coef_at_cutoff;
        eps   = P.eps;
        eps12 = eps * 12;
        debye = P.debye; inv_debye = P.inv_debye;
        abs_cut_sq = P.abs_cutoff * P.abs_cutoff;
        qi = pi.w; inv4pi = P.inv4pi;
        slot_p1 = t.slot_p1;
        // second per-slot parameter: LJ-family epsilon, HardCore core radius
        epsi  = (G == G_LJ || (G == G_EXV && kind == EXV_HARD_CORE)) ? t.slot_p1[slot] : 0.0;
        eps12f = (float)eps12; epsf = (float)eps; coefcf = (float)coefc;
        debf = (float)debye; invdf = (float)inv_debye;
        crsqf = (float)crsq; wif = (float)pi.w;
        fe = !NF && t.fe_energy != 0;
        force = a.force;
        slot_particle = t.slot_particle;
    }

    // Half lists (mixed form): the partner's share of the pair, the negated
    // fixed-point components of c r_ij.  Its own evaluation of the pair would
    // take r_ji = -r_ij exactly (an FP64 difference; the minimum image is odd
    // inside the cutoff), the same coefficient (every potential is symmetric
    // in its two parameters, and FP32 sums and products commute) and the same
    // rounding to the grid (round to nearest even is odd), so the integer sum
    // of each particle is the full lists' sum, bit for bit.
    // jp: the partner's particle when the caller has read it with its coordinates
    __device__ __forceinline__ void partner_add(double c, int q, double dx, double dy, double dz, int jp = -1) const
    {
        if constexpr(PREC == P_MIXED && NF && HALF)
        {
            if(c == 0.0) {return;}
            const long long x = fx_from_double(c * dx), y = fx_from_double(c * dy), z = fx_from_double(c * dz);
            unsigned long long* f =
                reinterpret_cast<unsigned long long*>(static_cast<longlong4*>(force) + (jp >= 0 ? jp : slot_particle[q]));
            if(x) {atomicAdd(f + 0, (unsigned long long)(-x));}
            if(y) {atomicAdd(f + 1, (unsigned long long)(-y));}
            if(z) {atomicAdd(f + 2, (unsigned long long)(-z));}
        }
    }

    // WCA, LennardJonesAttractive and UniformLennardJones through the generic
    // pair loop: f = r_ij (f_mag / |r|) with f_mag = potential.derivative(|r|),
    // a pair with f_mag = 0 skipped in the force pass; the energy-only pass
    // (calc_energy) sums potential(|r|) over every listed pair.  Formulas of
    // WCAPotential.hpp:37-58, LennardJonesAttractivePotential.hpp:36-70,
    // UniformLennardJonesPotential.hpp:41-61 (uniform sigma and epsilon are
    // equal per-slot values, which the Lorentz-Berthelot rule keeps as is).
    template<typename T>
    __device__ __forceinline__ static T fam_derivative(int kind, T r, T sigma, T epsilon, T cutoff_ratio)
    {
        if(kind == LJ_WCA)
        {
            if(sigma * T(SIXTH_ROOT_OF_TWO) < r) {return T(0);}
            const T rinv = T(1) / r;
            const T r1s1 = sigma * rinv;
            const T r3s3 = r1s1 * r1s1 * r1s1;
            const T r6s6 = r3s3 * r3s3;
            return T(24) * epsilon * (r6s6 * (T(1) - T(2) * r6s6)) * rinv;
        }
        if(kind == LJ_ATTRACTIVE)
        {
            if(r < sigma * T(SIXTH_ROOT_OF_TWO) || sigma * cutoff_ratio < r) {return T(0);}
            const T rinv = T(1) / r;
            const T sr1 = sigma * rinv;
            const T sr3 = sr1 * sr1 * sr1;
            const T sr6 = sr3 * sr3;
            return T(24) * epsilon * (sr6 - T(2) * sr6 * sr6) * rinv;
        }
        if(sigma * cutoff_ratio < r) {return T(0);}
        const T rinv = T(1) / r;
        const T sr1 = sigma * rinv;
        const T sr3 = sr1 * sr1 * sr1;
        const T sr6 = sr3 * sr3;
        return (epsilon * T(24)) * sr6 * (T(1) - T(2) * sr6) * rinv;
    }
    template<typename T>
    __device__ __forceinline__ static T fam_potential(int kind, T r, T sigma, T epsilon, T cutoff_ratio, T coefc)
    {
        if(kind == LJ_WCA)
        {
            if(sigma * T(SIXTH_ROOT_OF_TWO) < r) {return T(0);}
            const T r1s1 = sigma / r;
            const T r3s3 = r1s1 * r1s1 * r1s1;
            const T r6s6 = r3s3 * r3s3;
            return T(4) * epsilon * (r6s6 * (r6s6 - T(1)) + T(0.25));
        }
        if(kind == LJ_ATTRACTIVE)
        {
            if(r < sigma * T(SIXTH_ROOT_OF_TWO)) {return -epsilon;}
            if(sigma * cutoff_ratio < r) {return T(0);}
            const T sr1 = sigma / r;
            const T sr3 = sr1 * sr1 * sr1;
            const T sr6 = sr3 * sr3;
            return T(4) * epsilon * (sr6 * (sr6 - T(1)) - coefc);
        }
        if(sigma * cutoff_ratio < r) {return T(0);}
        const T sr1 = sigma / r;
        const T sr3 = sr1 * sr1 * sr1;
        const T sr6 = sr3 * sr3;
        return (epsilon * T(4)) * (sr6 * (sr6 - T(1)) - coefc);
    }
    __device__ __forceinline__ void family(int k, double sigma, double epsilon, double l2, double dx,
                                           double dy, double dz, bool count_e, Acc<PREC>& acc,
                                           double& energy, bool& ovf, int q, int jp) const
    {
        using T = typename std::conditional<PREC == P_FP64, double, float>::type;
        if(NF || fe)
        {
            const T rl = PREC == P_FP64 ? T(rsqrt(l2)) : T(rsqrtf((float)l2));
            const T l  = T(l2) * rl;
            const T f_mag = fam_derivative<T>(k, l, T(sigma), T(epsilon), T(cr));
            if(f_mag == T(0)) {return;}
            if(NF) {acc.add((double)(f_mag * rl), dx, dy, dz, ovf); partner_add((double)(f_mag * rl), q, dx, dy, dz, jp);}
            if(count_e) {energy += (double)fam_potential<T>(k, l, T(sigma), T(epsilon), T(cr), T(coefc));}
        }
        else if(count_e)
        {
            const T l = PREC == P_FP64 ? T(sqrt(l2)) : sqrtf((float)l2);
            energy += (double)fam_potential<T>(k, l, T(sigma), T(epsilon), T(cr), T(coefc));
        }
    }

    // InversePower (InversePowerPotential.hpp:38-57; sigma_ij = r_i + r_j)
    // and HardCoreExcludedVolume (HardCoreExcludedVolumePotential.hpp:44-80;
    // sigma_ij = s_i + s_j, R_ij = c_i + c_j) through the generic pair loop
    template<typename T>
    __device__ __forceinline__ T exv_derivative(T r, T sigma, T radius) const
    {
        if(kind == EXV_INVERSE_POWER)
        {
            if(sigma * T(cr) < r) {return T(0);}
            const T rinv = T(1) / r;
            const T d_r = sigma * rinv;
            const T drn = pow(d_r, T(power));
            return T(-power) * T(eps) * drn * rinv;
        }
        if(sigma * T(cr) + radius < r) {return T(0);}
        if(r < radius) {return T(INFINITY);}
        const T gapinv = T(1) / (r - radius);
        const T s1 = sigma * gapinv;
        const T s3 = s1 * s1 * s1;
        const T s6 = s3 * s3;
        return T(-12) * T(eps) * s6 * s6 * gapinv;
    }
    template<typename T>
    __device__ __forceinline__ T exv_potential(T r, T sigma, T radius) const
    {
        if(kind == EXV_INVERSE_POWER)
        {
            if(sigma * T(cr) < r) {return T(0);}
            const T d_r = sigma / r;
            const T drn = pow(d_r, T(power));
            return T(eps) * (drn - T(coefc));
        }
        if(sigma * T(cr) + radius < r) {return T(0);}
        if(r < radius) {return T(INFINITY);}
        const T gap = r - radius;
        const T s1 = sigma / gap;
        const T s3 = s1 * s1 * s1;
        const T s6 = s3 * s3;
        return T(eps) * (s6 * s6 - T(coefc));
    }
    __device__ __forceinline__ void exv_family(double sigma, double radius, double l2, double dx, double dy,
                                               double dz, bool count_e, Acc<PREC>& acc, double& energy,
                                               bool& ovf, int q, int jp) const
    {
        using T = typename std::conditional<PREC == P_FP64, double, float>::type;
        if(NF || fe)
        {
            const T rl = PREC == P_FP64 ? T(rsqrt(l2)) : T(rsqrtf((float)l2));
            const T l  = T(l2) * rl;
            const T f_mag = exv_derivative<T>(l, T(sigma), T(radius));
            if(f_mag == T(0)) {return;}
            if(NF) {acc.add((double)(f_mag * rl), dx, dy, dz, ovf); partner_add((double)(f_mag * rl), q, dx, dy, dz, jp);}
            if(count_e) {energy += (double)exv_potential<T>(l, T(sigma), T(radius));}
        }
        else if(count_e)
        {
            const T l = PREC == P_FP64 ? T(sqrt(l2)) : sqrtf((float)l2);
            energy += (double)exv_potential<T>(l, T(sigma), T(radius));
        }
    }

    __device__ __forceinline__ void operator()(const double4& pj, const int q, Acc<PREC>& acc,
                                               double& energy, bool& ovf, int jp = -1) const
    {
        double dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
        if(PER && periodic)
        {
            dx = min_image(dx, S->halfw[0], S->width[0]);
            dy = min_image(dy, S->halfw[1], S->width[1]);
            dz = min_image(dz, S->halfw[2], S->width[2]);
        }
        const double l2 = fma(dz, dz, fma(dy, dy, dx * dx));
        const bool count_e = NE && (s < q);
        if(G == G_EXV)
        {
            if(kind != EXV_PLAIN)
            {
                const double radius = kind == EXV_HARD_CORE ? epsi + slot_p1[q] : 0.0;
                exv_family(pi.w + pj.w, radius, l2, dx, dy, dz, count_e, acc, energy, ovf, q, jp);
                return;
            }
            const double sigma = pi.w + pj.w;
            const double sigma_sq = sigma * sigma;
            const bool in = !(sigma_sq * crsq < l2);
            if constexpr(PREC == P_FP64)
            {
                if(!in) {return;}
                const double rcp = 1.0 / l2;
                const double s2 = sigma_sq * rcp;
                const double s6 = s2 * s2 * s2;
                if(NF) {acc.add(-eps12 * s6 * s6 * rcp, dx, dy, dz, ovf);}
                if(count_e) {energy += eps * (s6 * s6 - coefc);}
            }
            else
            {
                // branch-free: every lane evaluates, pairs outside the
                // cutoff add an exact zero; sigma in FP32 from the two radii
                const float l2f = (float)l2;
                const float rcp = __frcp_rn(l2f);
                const float sg = wif + (float)pj.w;
                const float s2 = sg * sg * rcp;
                const float s6 = s2 * s2 * s2;
                const float cf = in ? -eps12f * s6 * s6 * rcp : 0.0f;
                if constexpr(NF)
                {
                    acc.add_c(cf, fabsf(cf) * fmaxf(l2f, 1.0f), dx, dy, dz, ovf);
                    partner_add((double)cf, q, dx, dy, dz, jp);
                }
                if(count_e && in) {energy += (double)(epsf * (s6 * s6 - coefcf));}
            }
        }
        else if(G == G_DH)
        {
            const bool in = l2 < abs_cut_sq;
            if constexpr(PREC == P_FP64)
            {
                if(!in) {return;}
                const double qq = (qi * pj.w) * inv4pi;     // symmetric in i, j
                const double rl = rsqrt(l2);
                const double l  = l2 * rl;
                const double ex = exp(-l * inv_debye);
                if(NF) {acc.add(-qq * (debye + l) * inv_debye / (l * l) * ex * rl, dx, dy, dz, ovf);}
                if(count_e) {energy += qq * (ex / l - coefc);}
            }
            else
            {
                // branch-free like ExcludedVolume: outside the cutoff the
                // distance is replaced by the cutoff and the force is zero
                // the charge product stays in FP64 and scales the FP32
                // coefficient of the unit-charge potential
                const double qq = (qi * pj.w) * inv4pi;
                const float l2f = in ? (float)l2 : (float)abs_cut_sq;
                const float rl = rsqrtf(l2f);
                const float l  = l2f * rl;
                const float ex = __expf(-l * invdf);
                const float cu = in ? -(debf + l) * invdf * (rl * rl) * ex * rl : 0.0f;
                if constexpr(NF)
                {
                    const float cf = (float)qq * cu;
                    acc.add_c(cf, fabsf(cf) * l, dx, dy, dz, ovf);
                    partner_add((double)cf, q, dx, dy, dz, jp);
                }
                if(count_e && in) {energy += qq * (double)(ex * rl - coefcf);}
            }
        }
        else   // G_LJ
        {
            const double sigma = (pi.w + pj.w) / 2;
            const double epsj = slot_p1[q];
            const double epsilon = (epsi == epsj) ? epsi : sqrt(epsi * epsj);
            if(kind != LJ_PLAIN)
            {
                family(kind, sigma, epsilon, l2, dx, dy, dz, count_e, acc, energy, ovf, q, jp);
                return;
            }
            const double sigma_sq = sigma * sigma;
            if(sigma_sq * crsq < l2) {return;}
            if constexpr(PREC == P_FP64)
            {
                const double rcp = 1.0 / l2;
                const double s2 = sigma_sq * rcp;
                const double s6 = s2 * s2 * s2;
                if(NF) {acc.add(24 * epsilon * (s6 - 2 * s6 * s6) * rcp, dx, dy, dz, ovf);}
                if(count_e) {energy += 4 * epsilon * (s6 * s6 - s6 - coefc);}
            }
            else
            {
                const float l2f = (float)l2;
                const float rcp = __frcp_rn(l2f);
                const float s2 = (float)sigma_sq * rcp;
                const float s6 = s2 * s2 * s2;
                const float ef = (float)epsilon;
                if constexpr(NF)
                {
                    const float cf = 24.0f * ef * (s6 - 2.0f * s6 * s6) * rcp;
                    acc.add_c(cf, fabsf(cf) * fmaxf(l2f, 1.0f), dx, dy, dz, ovf);
                    partner_add((double)cf, q, dx, dy, dz, jp);
                }
                if(count_e) {energy += (double)(4.0f * ef * (s6 * s6 - s6 - coefcf));}
            }
        }
    }
};

// List words PF_ROWS block rows ahead of the walk are requested into L2
// (prefetch.global.L2: no register, no wait), so that the walk's own loads of
// those words hit L2 instead of waiting on DRAM: a long list is a chain of
// dependent loads, and the rows a warp reads are np * TPP words apart.
constexpr int PF_ROWS = 8;
__device__ __forceinline__ void prefetch_l2(const void* p)
{
    asm volatile("prefetch.global.L2 [%0];" :: "l"(p));
}
// One request to the bulk copy engine for `bytes` (a multiple of 16) from p
// (16-byte aligned) into L2; nothing waits on it.
__device__ __forceinline__ void bulk_prefetch_l2(const void* p, unsigned bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(p), "r"(bytes) : "memory");
}

// One slot per TPP consecutive threads.  UNR: partners requested per batch.
// 1 keeps one partner in flight ahead of the pair being evaluated; 2 and 4
// issue the batch's list words, then its coordinates, before evaluating any
// of them (more loads in flight per thread, more registers).
// A slot's system and the number of partners its force launch walks (0 in a
// frozen system, which keeps its forces): the two loads are independent, the
// system's flag is read once they arrive, and only when the arena has a
// frozen system.
struct SlotHead {
    int sys;
    int n;
};
__device__ __forceinline__ SlotHead slot_head(const Arena& a, const TermArrays& t, long long s)
{
    const int sys = t.slot_sys[s];
    const int n = t.nnb[s];
    return {sys, a.any_frozen && a.sys[sys].frozen ? 0 : n};
}

// Counting sort of a block's slots by their list length (in units of `per`
// partners, 32 bins): returns the block-local index of the slot this group of
// threads takes, with that slot's head (read once by the group that loaded
// it, handed over in shared memory).  Slot numbering is unchanged; only
// which threads walk which list.  Every thread of the block must call it.
template<int GROUPS>
__device__ __forceinline__ int sorted_group(const Arena& a, const TermArrays& t, long long first_slot,
                                            int group, bool leader, int per, SlotHead& head)
{
    constexpr int NB = 32;
    __shared__ int bin_count[NB];
    __shared__ int perm[GROUPS];
    __shared__ SlotHead heads[GROUPS];
    if(threadIdx.x < NB) {bin_count[threadIdx.x] = 0;}
    const long long s = first_slot + group;
    SlotHead h{0, 0};
    if(leader && s < t.np) {h = slot_head(a, t, s);}
    __syncthreads();
    const int nb = (h.n + per - 1) / per;
    const int bin = nb < NB - 1 ? nb : NB - 1;
    const int rank = leader ? atomicAdd(&bin_count[bin], 1) : 0;
    if(leader) {heads[group] = h;}
    __syncthreads();
    if(threadIdx.x < 32)
    {
        const int v = bin_count[threadIdx.x];
        int incl = v;
#pragma unroll
        for(int o = 1; o < 32; o <<= 1)
        {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if((int)threadIdx.x >= o) {incl += y;}
        }
        bin_count[threadIdx.x] = incl - v;
    }
    __syncthreads();
    if(leader) {perm[bin_count[bin] + rank] = group;}
    __syncthreads();
    const int g = perm[group];
    head = heads[g];
    return g;
}

// Both pair kernels are held to 64 registers (four 256-thread blocks per SM):
// they wait on memory, and the occupancy is worth more than the few words
// spilled in the widest variants.
template<int PREC, int G, bool NF, bool NE, int TPP, bool PER, int UNR, bool SORT = false, bool HALF = false>
__global__ void __launch_bounds__(TPB, 4) k_pair(Arena a, TermArrays t)
{
    // TPP consecutive threads share one slot; lane lg walks partners lg,
    // lg + TPP, ... which the blocked list layout stores next to each other.
    // SORT: the block's groups take its slots in order of list length.
    const long long gt = (long long)blockIdx.x * TPB + threadIdx.x;
    long long s = gt / TPP;
    const int lg = (int)(threadIdx.x % TPP);
    SlotHead head{0, 0};
    if(SORT)
    {
        const long long first = (long long)blockIdx.x * (TPB / TPP);
        s = first + sorted_group<TPB / TPP>(a, t, first, (int)(threadIdx.x / TPP), lg == 0, TPP * UNR, head);
    }
    const bool active = s < t.np;
    if(!SORT && active) {head = slot_head(a, t, s);}
    const int sys = head.sys;
    double energy = 0.0;
    bool ovf = false;
    Acc<PREC> acc;
    if(active && head.n > 0)         // the group's slot; an empty list reads nothing
    {
        const PairEval<PREC, G, NF, NE, PER, HALF> eval(a, t, s, sys);
        const long long np = t.np;
        const int n = head.n;
        // word k = lg + r TPP of the slot's list: blocked layout, rows np TPP
        // words apart; slot-major layout, the slot's cap words in a row, the
        // whole list requested into L2 (16-byte aligned: cap is a multiple of
        // 32 words) before the walk starts
        const bool sm = t.slot_major != 0;
        const long long rs = sm ? TPP : np * TPP;
        const int* __restrict__ nbr = t.nbr + (sm ? s * t.cap : s * TPP) + lg;
        if(sm && lg == 0 && n > 0) {bulk_prefetch_l2(t.nbr + s * t.cap, (unsigned)((n + 3) / 4) * 16u);}
        const double4* __restrict__ pd = t.slot_pd;
        if(UNR == 1)
        {
            // software pipeline: the next partner's index and coordinates are
            // requested before the current pair is evaluated
            // the first list word is read whatever the list's length (every
            // slot owns cap >= TPP words), so that its load does not wait for
            // the length; a word past the length is never used as an index
            int k = lg;
            int q = __ldg(nbr);
            double4 pj = make_double4(0.0, 0.0, 0.0, 0.0);
            if(k < n) {pj = pd[q];}
            for(; k < n; k += TPP)
            {
                const int kn = k + TPP;
                const int kp = k + PF_ROWS * TPP;
                if(!sm && kp < n) {prefetch_l2(nbr + (long long)(kp / TPP) * rs);}
                int qn = q;
                double4 pn = pj;
                if(kn < n) {qn = __ldg(nbr + (long long)(kn / TPP) * rs); pn = pd[qn];}
                eval(pj, q, acc, energy, ovf);
                q = qn;
                pj = pn;
            }
        }
        else
        {
            for(int k = lg; k < n; k += UNR * TPP)
            {
                int qv[UNR];
                double4 pv[UNR];
#pragma unroll
                for(int u = 0; u < UNR; ++u)
                {
                    const int kp = k + (PF_ROWS + u) * TPP;
                    if(!sm && kp < n) {prefetch_l2(nbr + (long long)(kp / TPP) * rs);}
                }
#pragma unroll
                for(int u = 0; u < UNR; ++u)
                {
                    const int kk = k + u * TPP;
                    qv[u] = kk < n ? __ldg(nbr + (long long)(kk / TPP) * rs) : -1;
                }
#pragma unroll
                for(int u = 0; u < UNR; ++u) {pv[u] = qv[u] >= 0 ? pd[qv[u]] : eval.pi;}
#pragma unroll
                for(int u = 0; u < UNR; ++u) {if(qv[u] >= 0) {eval(pv[u], qv[u], acc, energy, ovf);}}
            }
        }
    }
    // group reduction: exact in fixed point, fixed order in FP64
#pragma unroll
    for(int o = TPP / 2; o > 0; o >>= 1) {acc.shfl_add(o);}
    if(active && NF && lg == 0) {acc.store(a.force, t.slot_particle[s]);}
    if(ovf) {atomicOr(&a.sys[sys].status, ST_FIXED_OVERFLOW);}
    if(NE)
    {
        const unsigned full = 0xffffffffu;
        const int s0 = __shfl_sync(full, sys, 0);
        const bool uniform = __all_sync(full, !active || sys == s0);
        if(uniform)
        {
            double e = energy;
#pragma unroll
            for(int o = 16; o > 0; o >>= 1) {e += __shfl_xor_sync(full, e, o);}
            if(__any_sync(full, active) && (threadIdx.x & 31) == 0) {atomicAdd(&a.sys[s0].energy[T_EXV + G], e);}
        }
        else if(active)
        {
            atomicAdd(&a.sys[sys].energy[T_EXV + G], energy);
        }
    }
}

// Block-vector schedule: one thread per slot reads its list L words at a
// time with one vector load (the blocked layout with L = tpp stores a slot's
// words k .. k + L - 1 next to each other, 4 L bytes aligned), the next block
// of words is requested before the current one is evaluated, and up to four
// partner coordinates are requested together.  A slot's list then costs one
// list latency per L partners instead of one per partner.
template<int L>
__device__ __forceinline__ void load_block(const int* __restrict__ p, int (&q)[L])
{
    if(L == 2)
    {
        const int2 v = __ldg(reinterpret_cast<const int2*>(p));
        q[0] = v.x; q[1] = v.y;
    }
    else
    {
#pragma unroll
        for(int c = 0; c < L / 4; ++c)
        {
            const int4 v = __ldg(reinterpret_cast<const int4*>(p) + c);
            q[4 * c] = v.x; q[4 * c + 1] = v.y; q[4 * c + 2] = v.z; q[4 * c + 3] = v.w;
        }
    }
}

// Schedules 2 and 3 (blocked list layout only).
// SORT: the block's threads take its 256 slots in order of their number of
// list blocks (a counting sort in shared memory), so that the lanes of a warp
// walk lists of about the same length; the slots themselves, and with them
// the spatial order of the partners, stay where they are.
template<int PREC, int G, bool PER, int L, bool SORT, bool HALF>
__global__ void __launch_bounds__(TPB, 4) k_pair_vec(Arena a, TermArrays t)
{
    long long s = (long long)blockIdx.x * TPB + threadIdx.x;
    SlotHead head{0, 0};
    if(SORT)
    {
        const long long first = (long long)blockIdx.x * TPB;
        s = first + sorted_group<TPB>(a, t, first, (int)threadIdx.x, true, L, head);
    }
    if(s >= t.np) {return;}
    if(!SORT) {head = slot_head(a, t, s);}
    if(head.n == 0) {return;}        // an empty list (frequent in half lists): nothing to add
    const int sys = head.sys;
    double energy = 0.0;
    bool ovf = false;
    Acc<PREC> acc;
    const PairEval<PREC, G, true, false, PER, HALF> eval(a, t, s, sys);
    const long long np = t.np;
    const int n = head.n;
    const double4* __restrict__ pd = t.slot_pd;
    constexpr int W = L < 4 ? L : 4;                 // partners requested together
    // the first block is read whatever the list's length (every slot owns
    // cap >= L words), so that its load does not wait for the length; words
    // past the length are never used as indices
    int q[L];
    load_block<L>(t.nbr + s * L, q);
    for(int k = 0; k < n; k += L)
    {
        int qn[L];
        if(k + L < n) {load_block<L>(t.nbr + ((long long)(k / L + 1) * np + s) * L, qn);}
        if(k + PF_ROWS * L < n) {prefetch_l2(t.nbr + ((long long)(k / L + PF_ROWS) * np + s) * L);}
        const int m = min(L, n - k);
#pragma unroll
        for(int u0 = 0; u0 < L; u0 += W)
        {
            double4 pv[W];
            int jv[W];                               // half lists: the partners' particles, read beside
#pragma unroll                                       // their coordinates, so the atomics wait on nothing
            for(int u = 0; u < W; ++u)
            {
                pv[u] = u0 + u < m ? pd[q[u0 + u]] : eval.pi;
                jv[u] = HALF && u0 + u < m ? t.slot_particle[q[u0 + u]] : -1;
            }
#pragma unroll
            for(int u = 0; u < W; ++u) {if(u0 + u < m) {eval(pv[u], q[u0 + u], acc, energy, ovf, jv[u]);}}
        }
#pragma unroll
        for(int u = 0; u < L; ++u) {q[u] = qn[u];}
    }
    acc.store(a.force, t.slot_particle[s]);
    if(ovf) {atomicOr(&a.sys[sys].status, ST_FIXED_OVERFLOW);}
}

// Warp-balanced schedule of the mixed form's force launch (schedule 1,
// blocked list layout only): a warp owns 32
// consecutive slots and splits the concatenation of their lists into 32 equal
// contiguous chunks, one per lane, so every lane evaluates the same number of
// pairs whatever the list lengths (one slot per thread leaves the lanes of
// short lists idle).  A lane sums the pairs of one slot in registers and adds
// the sum to the particle's fixed-point force with integer atomics when its
// chunk leaves that slot; integer sums are exact, so the result does not
// depend on where the chunks start.
template<int G, bool PER, int UNR, bool HALF>
__global__ void __launch_bounds__(TPB) k_pair_warp(Arena a, TermArrays t)
{
    __shared__ int seg[TPB / 32][33];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
    const long long gt = (long long)blockIdx.x * TPB + threadIdx.x;
    const long long s0 = gt - lane;                  // first slot of this warp
    int n_my = 0;
    if(gt < t.np)
    {
        n_my = slot_head(a, t, gt).n;                // 0 in a frozen system
    }
    int incl = n_my;
#pragma unroll
    for(int o = 1; o < 32; o <<= 1)
    {
        const int y = __shfl_up_sync(full, incl, o);
        if(lane >= o) {incl += y;}
    }
    seg[wl][lane] = incl - n_my;                     // first entry of slot s0 + lane
    if(lane == 31) {seg[wl][32] = incl;}
    __syncwarp();
    const int total = seg[wl][32];
    const int per = (total + 31) >> 5;
    int e = min(lane * per, total);
    const int e_end = min(e + per, total);
    if(e >= e_end) {return;}
    // slot of entry e: the last j with seg[j] <= e (seg is non-decreasing)
    int j = 0;
#pragma unroll
    for(int b = 16; b > 0; b >>= 1) {if(j + b < 32 && seg[wl][j + b] <= e) {j += b;}}

    const long long np = t.np;
    const int tpp = t.tpp;
    const int lt = __ffs(tpp) - 1;                   // tpp is a power of two
    const int* __restrict__ nbr = t.nbr;
    const double4* __restrict__ pd = t.slot_pd;
    while(e < e_end)
    {
        const long long s = s0 + j;
        const int b = seg[wl][j];
        const int kend = min(seg[wl][j + 1], e_end) - b;
        const int sys = t.slot_sys[s];
        const PairEval<P_MIXED, G, true, false, PER, HALF> eval(a, t, s, sys);
        Acc<P_MIXED> acc;
        double energy = 0.0;
        bool ovf = false;
        for(int k = e - b; k < kend; k += UNR)
        {
            int qv[UNR];
            double4 pv[UNR];
#pragma unroll
            for(int u = 0; u < UNR; ++u)
            {
                const int kk = k + u;
                qv[u] = kk < kend ? __ldg(nbr + (((long long)(kk >> lt) * np + s) << lt) + (kk & (tpp - 1))) : -1;
            }
#pragma unroll
            for(int u = 0; u < UNR; ++u) {pv[u] = qv[u] >= 0 ? pd[qv[u]] : eval.pi;}
#pragma unroll
            for(int u = 0; u < UNR; ++u) {if(qv[u] >= 0) {eval(pv[u], qv[u], acc, energy, ovf);}}
        }
        if(acc.x | acc.y | acc.z)
        {
            unsigned long long* f =
                reinterpret_cast<unsigned long long*>(static_cast<longlong4*>(a.force) + t.slot_particle[s]);
            atomicAdd(f + 0, (unsigned long long)acc.x);
            atomicAdd(f + 1, (unsigned long long)acc.y);
            atomicAdd(f + 2, (unsigned long long)acc.z);
        }
        if(ovf) {atomicOr(&a.sys[sys].status, ST_FIXED_OVERFLOW);}
        e = b + kend;
        ++j;
        while(j < 32 && seg[wl][j + 1] == seg[wl][j]) {++j;}     // skip empty lists
    }
}

// pairs (s < q) inside the potential's cutoff: the margin-free pair count
template<int G>
__global__ void k_count_cut(Arena a, TermArrays t, int sys_filter, unsigned long long* out)
{
    const long long s = (long long)blockIdx.x * 256 + threadIdx.x;
    unsigned long long cnt = 0;
    if(s < t.np && (sys_filter < 0 || t.slot_sys[s] == sys_filter))
    {
        const SysDev& S = a.sys[t.slot_sys[s]];
        const GlobalParams& P = S.g[G];
        const double4 pi = t.slot_pd[s];
        const int n = t.nnb[s];
        for(int k = 0; k < n; ++k)
        {
            const int q = t.nbr[nbr_pos(k, s, t.np, t.tpp, t.cap, t.slot_major)];
            if(q <= s) {continue;}
            const double4 pj = t.slot_pd[q];
            double dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
            if(S.boundary == B_PERIODIC)
            {
                dx = min_image(dx, S.halfw[0], S.width[0]);
                dy = min_image(dy, S.halfw[1], S.width[1]);
                dz = min_image(dz, S.halfw[2], S.width[2]);
            }
            const double l2 = fma(dz, dz, fma(dy, dy, dx * dx));
            bool in = false;
            if(G == G_EXV && P.kind == EXV_HARD_CORE)
            {
                const double sg = pi.w + pj.w, core = t.slot_p1[s] + t.slot_p1[q];
                in = !(sg * P.cutoff_ratio + core < sqrt(l2));
            }
            else if(G == G_EXV) {const double sg = pi.w + pj.w; in = !(sg * sg * P.cutoff_ratio_sq < l2);}
            else if(G == G_DH) {in = l2 < P.abs_cutoff * P.abs_cutoff;}
            else               {const double sg = (pi.w + pj.w) / 2; in = !(sg * sg * P.cutoff_ratio_sq < l2);}
            cnt += in ? 1 : 0;
        }
    }
#pragma unroll
    for(int o = 16; o > 0; o >>= 1) {cnt += __shfl_xor_sync(0xffffffffu, cnt, o);}
    if((threadIdx.x & 31) == 0 && cnt) {atomicAdd(out, cnt);}
}

template<int PREC, int G, int TPP, bool PER, bool HALF>
void dispatch_per(const Arena& a, TermArrays& t, bool nf, bool ne, cudaStream_t s)
{
    const unsigned nb = (unsigned)((t.np * TPP + TPB - 1) / TPB);
    if(nf && ne)  {k_pair<PREC, G, true,  true,  TPP, PER, 1><<<nb, TPB, 0, s>>>(a, t);}
    else if(nf)
    {
        // the per-step force launch: schedule and partner batch depth are tunable
        if constexpr(TPP > 1 && TPP <= 16)   // 32-word blocks: the slot-per-group kernel instead
        {
            if(t.schedule == 2 || t.schedule == 3)
            {
                const unsigned nv = (unsigned)((t.np + TPB - 1) / TPB);
                if(t.schedule == 3) {k_pair_vec<PREC, G, PER, TPP, true,  HALF><<<nv, TPB, 0, s>>>(a, t);}
                else                {k_pair_vec<PREC, G, PER, TPP, false, HALF><<<nv, TPB, 0, s>>>(a, t);}
                return;
            }
        }
        if(PREC == P_MIXED && t.schedule == 1)
        {
            const unsigned nw = (unsigned)((t.np + TPB - 1) / TPB);
            if(t.unroll == 4)      {k_pair_warp<G, PER, 4, HALF><<<nw, TPB, 0, s>>>(a, t);}
            else if(t.unroll == 2) {k_pair_warp<G, PER, 2, HALF><<<nw, TPB, 0, s>>>(a, t);}
            else                   {k_pair_warp<G, PER, 1, HALF><<<nw, TPB, 0, s>>>(a, t);}
        }
        else if(t.schedule == 4)
        {
            if(t.unroll == 4)      {k_pair<PREC, G, true, false, TPP, PER, 4, true, HALF><<<nb, TPB, 0, s>>>(a, t);}
            else if(t.unroll == 2) {k_pair<PREC, G, true, false, TPP, PER, 2, true, HALF><<<nb, TPB, 0, s>>>(a, t);}
            else                   {k_pair<PREC, G, true, false, TPP, PER, 1, true, HALF><<<nb, TPB, 0, s>>>(a, t);}
        }
        else if(t.unroll == 4) {k_pair<PREC, G, true, false, TPP, PER, 4, false, HALF><<<nb, TPB, 0, s>>>(a, t);}
        else if(t.unroll == 2) {k_pair<PREC, G, true, false, TPP, PER, 2, false, HALF><<<nb, TPB, 0, s>>>(a, t);}
        else                   {k_pair<PREC, G, true, false, TPP, PER, 1, false, HALF><<<nb, TPB, 0, s>>>(a, t);}
    }
    else if(ne)   {k_pair<PREC, G, false, true,  TPP, PER, 1><<<nb, TPB, 0, s>>>(a, t);}
}

template<int PREC, int G, int TPP, bool HALF>
void dispatch_tpp(const Arena& a, TermArrays& t, bool nf, bool ne, cudaStream_t s)
{
    if(t.any_periodic) {dispatch_per<PREC, G, TPP, true,  HALF>(a, t, nf, ne, s);}
    else               {dispatch_per<PREC, G, TPP, false, HALF>(a, t, nf, ne, s);}
}

// HALF: the mixed form's force launch on half lists (the partner's share
// added by the same evaluation); a template argument, so that the full-list
// kernels carry none of its code
template<int PREC, int G, bool HALF = false>
void dispatch(const Arena& a, TermArrays& t, bool nf, bool ne, cudaStream_t s)
{
    switch(t.tpp)
    {
        case 1:  dispatch_tpp<PREC, G, 1 , HALF>(a, t, nf, ne, s); break;
        case 2:  dispatch_tpp<PREC, G, 2 , HALF>(a, t, nf, ne, s); break;
        case 4:  dispatch_tpp<PREC, G, 4 , HALF>(a, t, nf, ne, s); break;
        case 8:  dispatch_tpp<PREC, G, 8 , HALF>(a, t, nf, ne, s); break;
        case 16: dispatch_tpp<PREC, G, 16, HALF>(a, t, nf, ne, s); break;
        default: dispatch_tpp<PREC, G, 32, HALF>(a, t, nf, ne, s); break;
    }
}

}  // namespace

void launch_gather(const Arena& a, TermArrays& t, cudaStream_t s)
{
    if(!t.on || t.np == 0) {return;}
    k_gather<<<(unsigned)((t.np + 255) / 256), 256, 0, s>>>(a, t);
    note_launches(1);
}

void launch_pair(const Arena& a, int g, TermArrays& t, bool need_force, bool need_energy,
                 int /*calc_energy_form*/, cudaStream_t s, bool gather)
{
    if(!t.on || t.np == 0) {return;}
    if(gather) {launch_gather(a, t, s);}
    note_launches(1);
    if(a.precision == P_FP64)
    {
        if(g == G_EXV)     {dispatch<P_FP64, G_EXV>(a, t, need_force, need_energy, s);}
        else if(g == G_DH) {dispatch<P_FP64, G_DH >(a, t, need_force, need_energy, s);}
        else               {dispatch<P_FP64, G_LJ >(a, t, need_force, need_energy, s);}
    }
    else
    {
        // mixed form: forces in FP32 with fixed-point sums (the per-step
        // path); energies, an observable read between steps, in the
        // reference's FP64 arithmetic
        if(need_force)
        {
            if(t.half)
            {
                if(g == G_EXV)     {dispatch<P_MIXED, G_EXV, true>(a, t, true, false, s);}
                else if(g == G_DH) {dispatch<P_MIXED, G_DH,  true>(a, t, true, false, s);}
                else               {dispatch<P_MIXED, G_LJ,  true>(a, t, true, false, s);}
            }
            else
            {
                if(g == G_EXV)     {dispatch<P_MIXED, G_EXV>(a, t, true, false, s);}
                else if(g == G_DH) {dispatch<P_MIXED, G_DH >(a, t, true, false, s);}
                else               {dispatch<P_MIXED, G_LJ >(a, t, true, false, s);}
            }
        }
        if(need_energy)
        {
            // with the forces: the energy of calc_force_and_energy
            TermArrays te = t;
            te.fe_energy = need_force ? 1 : 0;
            if(need_force) {note_launches(1);}
            if(g == G_EXV)     {dispatch<P_FP64, G_EXV>(a, te, false, true, s);}
            else if(g == G_DH) {dispatch<P_FP64, G_DH >(a, te, false, true, s);}
            else               {dispatch<P_FP64, G_LJ >(a, te, false, true, s);}
        }
    }
}

void launch_count_cut(const Arena& a, int g, TermArrays& t, int sys, unsigned long long* out,
                      cudaStream_t s)
{
    if(!t.on || t.np == 0) {return;}
    k_gather<<<(unsigned)((t.np + 255) / 256), 256, 0, s>>>(a, t);
    const unsigned nb = (unsigned)((t.np + 255) / 256);
    if(g == G_EXV)     {k_count_cut<G_EXV><<<nb, 256, 0, s>>>(a, t, sys, out);}
    else if(g == G_DH) {k_count_cut<G_DH ><<<nb, 256, 0, s>>>(a, t, sys, out);}
    else               {k_count_cut<G_LJ ><<<nb, 256, 0, s>>>(a, t, sys, out);}
    note_launches(2);
}

}  // namespace mjg
