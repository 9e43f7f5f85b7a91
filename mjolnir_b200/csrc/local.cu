// Local (bonded) terms, FP64 in both precision modes:
//   BondLength + Harmonic   forcefield/local/BondLengthInteraction.hpp:126-199,
//                           forcefield/local/HarmonicPotential.hpp:25-35 (V = k (v - v0)^2)
//   BondAngle  + Harmonic   forcefield/local/BondAngleInteraction.hpp:129-188
//   Dihedral   + Cosine     forcefield/local/DihedralAngleInteraction.hpp:157-227,
//                           forcefield/local/CosinePotential.hpp:29-39
// One thread per bond / angle / dihedral of every system; the forces land in
// the particles by atomics (FP64 atomics in the plain form, int64 fixed point
// in the mixed form, where the sum is exact and order independent).
#include "kernels.cuh"

namespace mjg {

namespace {

constexpr int TPB = 256;

template<int PREC>
__device__ __forceinline__ void add_force(void* force, int i, double fx, double fy, double fz)
{
    if(PREC == P_FP64)
    {
        double* f = reinterpret_cast<double*>(static_cast<double4*>(force) + i);
        atomicAdd(f + 0, fx); atomicAdd(f + 1, fy); atomicAdd(f + 2, fz);
    }
    else
    {
        unsigned long long* f = reinterpret_cast<unsigned long long*>(static_cast<longlong4*>(force) + i);
        atomicAdd(f + 0, (unsigned long long)fx_from_double(fx));
        atomicAdd(f + 1, (unsigned long long)fx_from_double(fy));
        atomicAdd(f + 2, (unsigned long long)fx_from_double(fz));
    }
}

__device__ __forceinline__ double3 direction(const SysDev& S, const double4& from, const double4& to)
{
    double3 d = make_double3(to.x - from.x, to.y - from.y, to.z - from.z);
    if(S.boundary == B_PERIODIC)
    {
        d.x = min_image(d.x, S.halfw[0], S.width[0]);
        d.y = min_image(d.y, S.halfw[1], S.width[1]);
        d.z = min_image(d.z, S.halfw[2], S.width[2]);
    }
    return d;
}
__device__ __forceinline__ double dot(double3 a, double3 b) {return a.x * b.x + a.y * b.y + a.z * b.z;}
__device__ __forceinline__ double3 cross(double3 a, double3 b)
{
    return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double clamp1(double x) {return fmin(fmax(x, -1.0), 1.0);}

__device__ __forceinline__ void reduce_energy(Arena& a, int sys, bool active, double e, int term)
{
    const unsigned full = 0xffffffffu;
    const int s0 = __shfl_sync(full, sys, 0);
    const bool uniform = __all_sync(full, !active || sys == s0);
    if(uniform)
    {
#pragma unroll
        for(int o = 16; o > 0; o >>= 1) {e += __shfl_xor_sync(full, e, o);}
        if(__any_sync(full, active) && (threadIdx.x & 31) == 0) {atomicAdd(&a.sys[s0].energy[term], e);}
    }
    else if(active)
    {
        atomicAdd(&a.sys[sys].energy[term], e);
    }
}

template<int PREC, bool NF, bool NE>
__global__ void __launch_bounds__(TPB) k_bonds(Arena a, LocalArrays l)
{
    const long long b = (long long)blockIdx.x * TPB + threadIdx.x;
    const bool active = b < l.nbond;
    const int sys = active ? l.bond_sys[b] : 0;
    double e = 0.0;
    if(active)
    {
        const SysDev& S = a.sys[sys];
        const int i0 = l.bond_idx[2 * b], i1 = l.bond_idx[2 * b + 1];
        const double k = l.bond_k[b], v0 = l.bond_v0[b];
        const double3 d = direction(S, a.pos[i0], a.pos[i1]);      // r1 - r0
        const double len2 = dot(d, d);
        const double rlen = rsqrt(len2);
        const double len  = len2 * rlen;
        const double dv   = len - v0;
        if(NE) {e = k * dv * dv;}
        if(NF)
        {
            const double c = -(2 * k * dv) * rlen;
            add_force<PREC>(a.force, i0, -d.x * c, -d.y * c, -d.z * c);
            add_force<PREC>(a.force, i1,  d.x * c,  d.y * c,  d.z * c);
        }
    }
    if(NE) {reduce_energy(a, sys, active, e, T_BOND);}
}

template<int PREC, bool NF, bool NE>
__global__ void __launch_bounds__(TPB) k_angles(Arena a, LocalArrays l)
{
    const long long b = (long long)blockIdx.x * TPB + threadIdx.x;
    const bool active = b < l.nangle;
    const int sys = active ? l.angle_sys[b] : 0;
    double e = 0.0;
    if(active)
    {
        const SysDev& S = a.sys[sys];
        const int i0 = l.angle_idx[3 * b], i1 = l.angle_idx[3 * b + 1], i2 = l.angle_idx[3 * b + 2];
        const double k = l.angle_k[b], v0 = l.angle_v0[b];
        const double4 p1 = a.pos[i1];
        const double3 r_ij = direction(S, p1, a.pos[i0]);
        const double3 r_kj = direction(S, p1, a.pos[i2]);
        const double inv_ij = rsqrt(dot(r_ij, r_ij));
        const double inv_kj = rsqrt(dot(r_kj, r_kj));
        const double3 eij = make_double3(r_ij.x * inv_ij, r_ij.y * inv_ij, r_ij.z * inv_ij);
        const double3 ekj = make_double3(r_kj.x * inv_kj, r_kj.y * inv_kj, r_kj.z * inv_kj);
        const double cos_t = clamp1(dot(eij, ekj));
        const double theta = acos(cos_t);
        const double dv = theta - v0;
        if(NE) {e = k * dv * dv;}
        if(NF)
        {
            const double coef = -(2 * k * dv);
            const double sin_t = sin(theta);
            const double cis = coef / fmax(sin_t, 1e-8);          // math/constants.hpp:26
            const double ci = cis * inv_ij, ck = cis * inv_kj;
            const double3 Fi = make_double3(ci * (cos_t * eij.x - ekj.x), ci * (cos_t * eij.y - ekj.y), ci * (cos_t * eij.z - ekj.z));
            const double3 Fk = make_double3(ck * (cos_t * ekj.x - eij.x), ck * (cos_t * ekj.y - eij.y), ck * (cos_t * ekj.z - eij.z));
            add_force<PREC>(a.force, i0, Fi.x, Fi.y, Fi.z);
            add_force<PREC>(a.force, i1, -Fi.x - Fk.x, -Fi.y - Fk.y, -Fi.z - Fk.z);
            add_force<PREC>(a.force, i2, Fk.x, Fk.y, Fk.z);
        }
    }
    if(NE) {reduce_energy(a, sys, active, e, T_ANGLE);}
}

template<int PREC, bool NF, bool NE>
__global__ void __launch_bounds__(TPB) k_dihedrals(Arena a, LocalArrays l)
{
    const long long b = (long long)blockIdx.x * TPB + threadIdx.x;
    const bool active = b < l.ndihd;
    const int sys = active ? l.dihd_sys[b] : 0;
    double e = 0.0;
    if(active)
    {
        const SysDev& S = a.sys[sys];
        const int i0 = l.dihd_idx[4 * b], i1 = l.dihd_idx[4 * b + 1];
        const int i2 = l.dihd_idx[4 * b + 2], i3 = l.dihd_idx[4 * b + 3];
        const double K = l.dihd_k[b], v0 = l.dihd_v0[b];
        const double nn = (double)l.dihd_n[b];
        const double4 rj = a.pos[i1], rk = a.pos[i2];
        const double3 r_ij = direction(S, rj, a.pos[i0]);
        const double3 r_kj = direction(S, rj, rk);
        const double3 r_lk = direction(S, rk, a.pos[i3]);
        const double3 r_kl = make_double3(-r_lk.x, -r_lk.y, -r_lk.z);
        const double r_kj_lensq  = dot(r_kj, r_kj);
        const double r_kj_rlen   = rsqrt(r_kj_lensq);
        const double r_kj_rlensq = r_kj_rlen * r_kj_rlen;
        const double r_kj_len    = r_kj_rlen * r_kj_lensq;
        const double3 m = cross(r_ij, r_kj);
        const double3 n = cross(r_kj, r_kl);
        const double m_lensq = dot(m, m);
        const double n_lensq = dot(n, n);
        const double cos_phi = clamp1(dot(m, n) * rsqrt(m_lensq * n_lensq));
        const double phi = copysign(acos(cos_phi), dot(r_ij, n));
        const double dv = phi - v0;
        if(NE) {e = K * (1 + cos(nn * dv));}
        if(NF)
        {
            const double coef = K * nn * sin(nn * dv);                // -dV/dphi
            const double cfi =  coef * r_kj_len / m_lensq;
            const double cfl = -coef * r_kj_len / n_lensq;
            const double3 Fi = make_double3(cfi * m.x, cfi * m.y, cfi * m.z);
            const double3 Fl = make_double3(cfl * n.x, cfl * n.y, cfl * n.z);
            const double cijk = dot(r_ij, r_kj) * r_kj_rlensq;
            const double cjkl = dot(r_kl, r_kj) * r_kj_rlensq;
            add_force<PREC>(a.force, i0, Fi.x, Fi.y, Fi.z);
            add_force<PREC>(a.force, i1, (cijk - 1.0) * Fi.x - cjkl * Fl.x, (cijk - 1.0) * Fi.y - cjkl * Fl.y,
                            (cijk - 1.0) * Fi.z - cjkl * Fl.z);
            add_force<PREC>(a.force, i2, (cjkl - 1.0) * Fl.x - cijk * Fi.x, (cjkl - 1.0) * Fl.y - cijk * Fi.y,
                            (cjkl - 1.0) * Fl.z - cijk * Fi.z);
            add_force<PREC>(a.force, i3, Fl.x, Fl.y, Fl.z);
        }
    }
    if(NE) {reduce_energy(a, sys, active, e, T_DIHEDRAL);}
}

template<int PREC, bool NF, bool NE>
void run_all(const Arena& a, const LocalArrays& l, int mask, cudaStream_t s)
{
    if((mask & 1) && l.nbond  > 0) {k_bonds    <PREC, NF, NE><<<(unsigned)((l.nbond  + TPB - 1) / TPB), TPB, 0, s>>>(a, l); note_launches(1);}
    if((mask & 2) && l.nangle > 0) {k_angles   <PREC, NF, NE><<<(unsigned)((l.nangle + TPB - 1) / TPB), TPB, 0, s>>>(a, l); note_launches(1);}
    if((mask & 4) && l.ndihd  > 0) {k_dihedrals<PREC, NF, NE><<<(unsigned)((l.ndihd  + TPB - 1) / TPB), TPB, 0, s>>>(a, l); note_launches(1);}
}

}  // namespace

void launch_local(const Arena& a, const LocalArrays& l, int mask, bool nf, bool ne,
                  int /*calc_energy_form*/, cudaStream_t s)
{
    if(a.precision == P_FP64)
    {
        if(nf && ne) {run_all<P_FP64, true, true>(a, l, mask, s);}
        else if(nf)  {run_all<P_FP64, true, false>(a, l, mask, s);}
        else if(ne)  {run_all<P_FP64, false, true>(a, l, mask, s);}
    }
    else
    {
        if(nf && ne) {run_all<P_MIXED, true, true>(a, l, mask, s);}
        else if(nf)  {run_all<P_MIXED, true, false>(a, l, mask, s);}
        else if(ne)  {run_all<P_MIXED, false, true>(a, l, mask, s);}
    }
}

}  // namespace mjg
