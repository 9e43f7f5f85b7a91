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
    __device__ __forceinline__ void shfl_add(int o)
    {
        x += __shfl_xor_sync(0xffffffffu, x, o);
        y += __shfl_xor_sync(0xffffffffu, y, o);
        z += __shfl_xor_sync(0xffffffffu, z, o);
    }
    __device__ __forceinline__ void store(void* force, long long i) const
    {
        longlong4* f = static_cast<longlong4*>(force) + i;
        longlong4 v = *f;
        v.x += x; v.y += y; v.z += z;
        *f = v;
    }
};

// PER: some system of the arena is periodic (the minimum image is applied
// where the system asks for it); without it the image code is compiled out.
template<int PREC, int G, bool NF, bool NE, int TPP, bool PER>
__global__ void __launch_bounds__(TPB) k_pair(Arena a, TermArrays t)
{
    // TPP consecutive threads share one slot; lane lg walks partners lg,
    // lg + TPP, ... which the blocked list layout stores next to each other
    const long long gt = (long long)blockIdx.x * TPB + threadIdx.x;
    const long long s = gt / TPP;
    const int lg = (int)(threadIdx.x % TPP);
    const bool active = s < t.np;
    const int sys = active ? t.slot_sys[s] : 0;
    double energy = 0.0;
    bool ovf = false;
    Acc<PREC> acc;
    if(active)
    {
        const SysDev& S = a.sys[sys];
        const GlobalParams& P = S.g[G];
        const bool periodic = PER && S.boundary == B_PERIODIC;
        const double4 pi = t.slot_pd[s];
        const long long np = t.np;
        const int n = S.frozen ? 0 : t.nnb[s];       // a frozen system keeps its forces

        // potential constants
        const double crsq  = P.cutoff_ratio_sq;
        const double coefc = P.coef_at_cutoff;
        const double eps   = P.eps;
        const double eps12 = eps * 12;
        const double debye = P.debye, inv_debye = P.inv_debye, abs_cut = P.abs_cutoff;
        const double abs_cut_sq = abs_cut * abs_cut;
        const double qi = pi.w, inv4pi = P.inv4pi;
        const double epsi  = (G == G_LJ) ? t.slot_p1[s] : 0.0;
        const float  eps12f = (float)eps12, epsf = (float)eps, coefcf = (float)coefc;
        const float  debf = (float)debye, invdf = (float)inv_debye;
        const int* __restrict__ nbr = t.nbr + s * TPP + lg;
        const double4* __restrict__ pd = t.slot_pd;

        // software pipeline: the next partner's index and coordinates are
        // requested before the current pair is evaluated
        int k = lg;
        int q = 0;
        double4 pj = make_double4(0.0, 0.0, 0.0, 0.0);
        if(k < n) {q = __ldg(nbr + (long long)(k / TPP) * np * TPP); pj = pd[q];}
        for(; k < n; k += TPP)
        {
            const int kn = k + TPP;
            int qn = q;
            double4 pn = pj;
            if(kn < n) {qn = __ldg(nbr + (long long)(kn / TPP) * np * TPP); pn = pd[qn];}
            do {
            double dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
            if(PER && periodic)
            {
                dx = min_image(dx, S.halfw[0], S.width[0]);
                dy = min_image(dy, S.halfw[1], S.width[1]);
                dz = min_image(dz, S.halfw[2], S.width[2]);
            }
            const double l2 = fma(dz, dz, fma(dy, dy, dx * dx));
            const bool count_e = NE && (s < q);
            if(G == G_EXV)
            {
                const double sigma = pi.w + pj.w;
                const double sigma_sq = sigma * sigma;
                const bool in = !(sigma_sq * crsq < l2);
                if(PREC == P_FP64)
                {
                    if(!in) {break;}
                    const double rcp = 1.0 / l2;
                    const double s2 = sigma_sq * rcp;
                    const double s6 = s2 * s2 * s2;
                    if(NF) {acc.add(-eps12 * s6 * s6 * rcp, dx, dy, dz, ovf);}
                    if(count_e) {energy += eps * (s6 * s6 - coefc);}
                }
                else
                {
                    // branch-free: every lane evaluates, pairs outside the
                    // cutoff add an exact zero
                    const float rcp = __frcp_rn((float)l2);
                    const float s2 = (float)sigma_sq * rcp;
                    const float s6 = s2 * s2 * s2;
                    const float cf = in ? -eps12f * s6 * s6 * rcp : 0.0f;
                    if(NF) {acc.add((double)cf, dx, dy, dz, ovf);}
                    if(count_e && in) {energy += (double)(epsf * (s6 * s6 - coefcf));}
                }
            }
            else if(G == G_DH)
            {
                if(!(l2 < abs_cut_sq)) {break;}
                if(PREC == P_FP64)
                {
                    const double qq = (qi * pj.w) * inv4pi;     // symmetric in i, j
                    const double rl = rsqrt(l2);
                    const double l  = l2 * rl;
                    const double ex = exp(-l * inv_debye);
                    if(NF) {acc.add(-qq * (debye + l) * inv_debye / (l * l) * ex * rl, dx, dy, dz, ovf);}
                    if(count_e) {energy += qq * (ex / l - coefc);}
                }
                else
                {
                    const float qq = (float)((qi * pj.w) * inv4pi);
                    const float l2f = (float)l2;
                    const float rl = rsqrtf(l2f);
                    const float l  = l2f * rl;
                    const float ex = __expf(-l * invdf);
                    if(NF) {acc.add((double)(-qq * (debf + l) * invdf * (rl * rl) * ex * rl), dx, dy, dz, ovf);}
                    if(count_e) {energy += (double)(qq * (ex * rl - coefcf));}
                }
            }
            else   // G_LJ
            {
                const double sigma = (pi.w + pj.w) / 2;
                const double epsj = t.slot_p1[q];
                const double epsilon = (epsi == epsj) ? epsi : sqrt(epsi * epsj);
                const double sigma_sq = sigma * sigma;
                if(sigma_sq * crsq < l2) {break;}
                if(PREC == P_FP64)
                {
                    const double rcp = 1.0 / l2;
                    const double s2 = sigma_sq * rcp;
                    const double s6 = s2 * s2 * s2;
                    if(NF) {acc.add(24 * epsilon * (s6 - 2 * s6 * s6) * rcp, dx, dy, dz, ovf);}
                    if(count_e) {energy += 4 * epsilon * (s6 * s6 - s6 - coefc);}
                }
                else
                {
                    const float rcp = __frcp_rn((float)l2);
                    const float s2 = (float)sigma_sq * rcp;
                    const float s6 = s2 * s2 * s2;
                    const float ef = (float)epsilon;
                    if(NF) {acc.add((double)(24.0f * ef * (s6 - 2.0f * s6 * s6) * rcp), dx, dy, dz, ovf);}
                    if(count_e) {energy += (double)(4.0f * ef * (s6 * s6 - s6 - coefcf));}
                }
            }
            } while(0);
            q = qn;
            pj = pn;

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
            const int q = t.nbr[nbr_index(k, s, t.np, t.tpp)];
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
            if(G == G_EXV)     {const double sg = pi.w + pj.w; in = !(sg * sg * P.cutoff_ratio_sq < l2);}
            else if(G == G_DH) {in = l2 < P.abs_cutoff * P.abs_cutoff;}
            else               {const double sg = (pi.w + pj.w) / 2; in = !(sg * sg * P.cutoff_ratio_sq < l2);}
            cnt += in ? 1 : 0;
        }
    }
#pragma unroll
    for(int o = 16; o > 0; o >>= 1) {cnt += __shfl_xor_sync(0xffffffffu, cnt, o);}
    if((threadIdx.x & 31) == 0 && cnt) {atomicAdd(out, cnt);}
}

template<int PREC, int G, int TPP, bool PER>
void dispatch_per(const Arena& a, TermArrays& t, bool nf, bool ne, cudaStream_t s)
{
    const unsigned nb = (unsigned)((t.np * TPP + TPB - 1) / TPB);
    if(nf && ne)  {k_pair<PREC, G, true,  true,  TPP, PER><<<nb, TPB, 0, s>>>(a, t);}
    else if(nf)   {k_pair<PREC, G, true,  false, TPP, PER><<<nb, TPB, 0, s>>>(a, t);}
    else if(ne)   {k_pair<PREC, G, false, true,  TPP, PER><<<nb, TPB, 0, s>>>(a, t);}
}

template<int PREC, int G, int TPP>
void dispatch_tpp(const Arena& a, TermArrays& t, bool nf, bool ne, cudaStream_t s)
{
    if(t.any_periodic) {dispatch_per<PREC, G, TPP, true >(a, t, nf, ne, s);}
    else               {dispatch_per<PREC, G, TPP, false>(a, t, nf, ne, s);}
}

template<int PREC, int G>
void dispatch(const Arena& a, TermArrays& t, bool nf, bool ne, cudaStream_t s)
{
    switch(t.tpp)
    {
        case 1:  dispatch_tpp<PREC, G, 1 >(a, t, nf, ne, s); break;
        case 2:  dispatch_tpp<PREC, G, 2 >(a, t, nf, ne, s); break;
        case 4:  dispatch_tpp<PREC, G, 4 >(a, t, nf, ne, s); break;
        case 8:  dispatch_tpp<PREC, G, 8 >(a, t, nf, ne, s); break;
        default: dispatch_tpp<PREC, G, 16>(a, t, nf, ne, s); break;
    }
}

}  // namespace

void launch_pair(const Arena& a, int g, TermArrays& t, bool need_force, bool need_energy,
                 int /*calc_energy_form*/, cudaStream_t s)
{
    if(!t.on || t.np == 0) {return;}
    k_gather<<<(unsigned)((t.np + 255) / 256), 256, 0, s>>>(a, t);
    note_launches(2);
    if(a.precision == P_FP64)
    {
        if(g == G_EXV)     {dispatch<P_FP64, G_EXV>(a, t, need_force, need_energy, s);}
        else if(g == G_DH) {dispatch<P_FP64, G_DH >(a, t, need_force, need_energy, s);}
        else               {dispatch<P_FP64, G_LJ >(a, t, need_force, need_energy, s);}
    }
    else
    {
        if(g == G_EXV)     {dispatch<P_MIXED, G_EXV>(a, t, need_force, need_energy, s);}
        else if(g == G_DH) {dispatch<P_MIXED, G_DH >(a, t, need_force, need_energy, s);}
        else               {dispatch<P_MIXED, G_LJ >(a, t, need_force, need_energy, s);}
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
