// Local (bonded) terms; the FP64 form keeps the reference's formulas, the
// mixed form evaluates them in FP32 from FP64 displacements, and with the
// FP64 formulas where a bond angle is within 11.5 degrees of collinear (see
// below):
//   BondLength + Harmonic   forcefield/local/BondLengthInteraction.hpp:126-199,
//                           forcefield/local/HarmonicPotential.hpp:25-35 (V = k (v - v0)^2)
//   BondAngle  + Harmonic   forcefield/local/BondAngleInteraction.hpp:129-188
//   Dihedral   + Cosine     forcefield/local/DihedralAngleInteraction.hpp:157-227,
//                           forcefield/local/CosinePotential.hpp:29-39
// One fused launch: one thread per bond / angle / dihedral of every system;
// the forces are summed per block in shared memory and land in the particles
// by atomics (FP64 atomics in the plain form, int64 fixed point in the mixed
// form, where the sum is exact and order independent).
#include "kernels.cuh"

namespace mjg {

namespace {

constexpr int TPB = 256;

// Forces of one block's terms are summed in shared memory over a window of
// WINDOW particles starting at the block's first particle (bonds, angles and
// dihedrals of a chain touch a narrow index range), then added to global
// memory once per particle; a particle outside the window goes to global
// memory directly.
constexpr int SEG = 256;              // particles owned by one block (window start)
constexpr int HALO = 64;              // terms may reach this far past the window
constexpr int WINDOW = SEG + HALO;

template<int PREC> struct WinT;
template<> struct WinT<P_FP64>  {using type = double;};
template<> struct WinT<P_MIXED> {using type = unsigned long long;};

template<int PREC>
struct Window {
    using T = typename WinT<PREC>::type;
    T* w;         // [3 * WINDOW] in shared memory
    int base;
    __device__ __forceinline__ void add(void* force, int i, double fx, double fy, double fz)
    {
        const int k = i - base;
        if(k >= 0 && k < WINDOW)
        {
            if(PREC == P_FP64)
            {
                atomicAdd(reinterpret_cast<double*>(w) + 3 * k + 0, fx);
                atomicAdd(reinterpret_cast<double*>(w) + 3 * k + 1, fy);
                atomicAdd(reinterpret_cast<double*>(w) + 3 * k + 2, fz);
            }
            else
            {
                atomicAdd(reinterpret_cast<unsigned long long*>(w) + 3 * k + 0, (unsigned long long)fx_from_double(fx));
                atomicAdd(reinterpret_cast<unsigned long long*>(w) + 3 * k + 1, (unsigned long long)fx_from_double(fy));
                atomicAdd(reinterpret_cast<unsigned long long*>(w) + 3 * k + 2, (unsigned long long)fx_from_double(fz));
            }
            return;
        }
        global_add(force, i, fx, fy, fz);
    }
    __device__ __forceinline__ static void global_add(void* force, int i, double fx, double fy, double fz)
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
    __device__ __forceinline__ void flush(void* force, long long n) const
    {
        for(int k = threadIdx.x; k < WINDOW; k += blockDim.x)
        {
            const long long i = (long long)base + k;
            if(i >= n) {break;}
            const T x = w[3 * k], y = w[3 * k + 1], z = w[3 * k + 2];
            if(x == T(0) && y == T(0) && z == T(0)) {continue;}
            if(PREC == P_FP64)
            {
                double* f = reinterpret_cast<double*>(static_cast<double4*>(force) + i);
                atomicAdd(f + 0, (double)x); atomicAdd(f + 1, (double)y); atomicAdd(f + 2, (double)z);
            }
            else
            {
                unsigned long long* f = reinterpret_cast<unsigned long long*>(static_cast<longlong4*>(force) + i);
                atomicAdd(f + 0, (unsigned long long)x); atomicAdd(f + 1, (unsigned long long)y);
                atomicAdd(f + 2, (unsigned long long)z);
            }
        }
    }
};

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
__device__ __forceinline__ void do_bond(Arena& a, const LocalArrays& l, long long b, bool active,
                                         Window<PREC>& W)
{
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
            W.add(a.force, i0, -d.x * c, -d.y * c, -d.z * c);
            W.add(a.force, i1,  d.x * c,  d.y * c,  d.z * c);
        }
    }
    if(NE) {reduce_energy(a, sys, active, e, T_BOND);}
}

// the reference's formulas for one (active) angle: adds its forces, returns
// its energy (NE)
template<int PREC, bool NF, bool NE>
__device__ __forceinline__ double angle_fp64(Arena& a, const LocalArrays& l, long long b, Window<PREC>& W)
{
    double e = 0.0;
    const SysDev& S = a.sys[l.angle_sys[b]];
    {
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
            W.add(a.force, i0, Fi.x, Fi.y, Fi.z);
            W.add(a.force, i1, -Fi.x - Fk.x, -Fi.y - Fk.y, -Fi.z - Fk.z);
            W.add(a.force, i2, Fk.x, Fk.y, Fk.z);
        }
    }
    return e;
}

template<int PREC, bool NF, bool NE>
__device__ __forceinline__ void do_angle(Arena& a, const LocalArrays& l, long long b, bool active,
                                         Window<PREC>& W)
{
    const int sys = active ? l.angle_sys[b] : 0;
    const double e = active ? angle_fp64<PREC, NF, NE>(a, l, b, W) : 0.0;
    if(NE) {reduce_energy(a, sys, active, e, T_ANGLE);}
}

// the reference's formulas for one (active) dihedral: adds its forces,
// returns its energy (NE)
template<int PREC, bool NF, bool NE>
__device__ __forceinline__ double dihedral_fp64(Arena& a, const LocalArrays& l, long long b, Window<PREC>& W)
{
    double e = 0.0;
    const SysDev& S = a.sys[l.dihd_sys[b]];
    {
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
            W.add(a.force, i0, Fi.x, Fi.y, Fi.z);
            W.add(a.force, i1, (cijk - 1.0) * Fi.x - cjkl * Fl.x, (cijk - 1.0) * Fi.y - cjkl * Fl.y,
                            (cijk - 1.0) * Fi.z - cjkl * Fl.z);
            W.add(a.force, i2, (cjkl - 1.0) * Fl.x - cijk * Fi.x, (cjkl - 1.0) * Fl.y - cijk * Fi.y,
                            (cjkl - 1.0) * Fl.z - cijk * Fi.z);
            W.add(a.force, i3, Fl.x, Fl.y, Fl.z);
        }
    }
    return e;
}

template<int PREC, bool NF, bool NE>
__device__ __forceinline__ void do_dihedral(Arena& a, const LocalArrays& l, long long b, bool active,
                                         Window<PREC>& W)
{
    const int sys = active ? l.dihd_sys[b] : 0;
    const double e = active ? dihedral_fp64<PREC, NF, NE>(a, l, b, W) : 0.0;
    if(NE) {reduce_energy(a, sys, active, e, T_DIHEDRAL);}
}

// ----------------------------------------------------------- mixed form
// sin of a bond angle below which an angle or dihedral is evaluated with the
// FP64 formulas instead (ill-conditioned in FP32)
constexpr float ILL_SIN = 0.2f;
// The same terms in FP32 from FP64 displacements: bond stretch via
// (r^2 - v0^2) / (r + v0) with r^2 - v0^2 in FP64, the angle from atan2 of the
// cross and dot products, the dihedral from (cos phi, sin phi) of the normals
// (phi = atan2(|r_kj| r_ij.n, m.n) has the reference's sign convention) and
// cos / sin of n (phi - v0) by the multiple-angle recurrence, so no FP64
// transcendental is evaluated.  Parameters come pre-packed as floats.

__device__ __forceinline__ float3 fdir(const SysDev& S, const double4& from, const double4& to)
{
    const double3 d = direction(S, from, to);
    return make_float3((float)d.x, (float)d.y, (float)d.z);
}
__device__ __forceinline__ float fdot(float3 a, float3 b) {return a.x * b.x + a.y * b.y + a.z * b.z;}
__device__ __forceinline__ float3 fcross(float3 a, float3 b)
{
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

template<int PREC, bool NF, bool NE>
__device__ __forceinline__ void do_bond_f32(Arena& a, const LocalArrays& l, long long b, bool active,
                                            Window<PREC>& W)
{
    const int sys = active ? l.bond_sys[b] : 0;
    double e = 0.0;
    if(active)
    {
        const SysDev& S = a.sys[sys];
        const int i0 = l.bond_idx[2 * b], i1 = l.bond_idx[2 * b + 1];
        const float2 kv = l.bond_kv[b];
        const double3 d = direction(S, a.pos[i0], a.pos[i1]);
        const double len2 = dot(d, d);
        const float lenf = sqrtf((float)len2);
        const float dv = (float)(len2 - (double)kv.y * (double)kv.y) / (lenf + kv.y);
        if(NE) {e = (double)(kv.x * dv * dv);}
        if(NF)
        {
            const double c = (double)(-(2.0f * kv.x * dv) / lenf);
            W.add(a.force, i0, -d.x * c, -d.y * c, -d.z * c);
            W.add(a.force, i1,  d.x * c,  d.y * c,  d.z * c);
        }
    }
    if(NE) {reduce_energy(a, sys, active, e, T_BOND);}
}

template<int PREC, bool NF, bool NE>
__device__ __forceinline__ void do_angle_f32(Arena& a, const LocalArrays& l, long long b, bool active,
                                             Window<PREC>& W)
{
    const int sys = active ? l.angle_sys[b] : 0;
    double e = 0.0;
    if(active)
    {
        const SysDev& S = a.sys[sys];
        const int i0 = l.angle_idx[3 * b], i1 = l.angle_idx[3 * b + 1], i2 = l.angle_idx[3 * b + 2];
        const float2 kv = l.angle_kv[b];
        const double4 p1 = a.pos[i1];
        const float3 rij = fdir(S, p1, a.pos[i0]);
        const float3 rkj = fdir(S, p1, a.pos[i2]);
        const float inv_ij = rsqrtf(fdot(rij, rij));
        const float inv_kj = rsqrtf(fdot(rkj, rkj));
        const float3 eij = make_float3(rij.x * inv_ij, rij.y * inv_ij, rij.z * inv_ij);
        const float3 ekj = make_float3(rkj.x * inv_kj, rkj.y * inv_kj, rkj.z * inv_kj);
        const float3 cr = fcross(eij, ekj);
        const float sin_t = sqrtf(fdot(cr, cr));
        if(sin_t < ILL_SIN)
        {
            // within 11.5 degrees of collinear the FP32 cross products and
            // differences of unit vectors lose the force: the FP64 formulas
            e = angle_fp64<PREC, NF, NE>(a, l, b, W);
        }
        else
        {
            const float cos_t = fdot(eij, ekj);
            const float theta = atan2f(sin_t, cos_t);
            const float dv = theta - kv.y;
            if(NE) {e = (double)(kv.x * dv * dv);}
            if(NF)
            {
                const float cis = -(2.0f * kv.x * dv) / fmaxf(sin_t, 1e-8f);
                const float ci = cis * inv_ij, ck = cis * inv_kj;
                const float cc = fminf(fmaxf(cos_t, -1.0f), 1.0f);
                const double3 Fi = make_double3(ci * (cc * eij.x - ekj.x), ci * (cc * eij.y - ekj.y), ci * (cc * eij.z - ekj.z));
                const double3 Fk = make_double3(ck * (cc * ekj.x - eij.x), ck * (cc * ekj.y - eij.y), ck * (cc * ekj.z - eij.z));
                W.add(a.force, i0, Fi.x, Fi.y, Fi.z);
                W.add(a.force, i1, -Fi.x - Fk.x, -Fi.y - Fk.y, -Fi.z - Fk.z);
                W.add(a.force, i2, Fk.x, Fk.y, Fk.z);
            }
        }
    }
    if(NE) {reduce_energy(a, sys, active, e, T_ANGLE);}
}

template<int PREC, bool NF, bool NE>
__device__ __forceinline__ void do_dihedral_f32(Arena& a, const LocalArrays& l, long long b, bool active,
                                                Window<PREC>& W)
{
    const int sys = active ? l.dihd_sys[b] : 0;
    double e = 0.0;
    if(active)
    {
        const SysDev& S = a.sys[sys];
        const int i0 = l.dihd_idx[4 * b], i1 = l.dihd_idx[4 * b + 1];
        const int i2 = l.dihd_idx[4 * b + 2], i3 = l.dihd_idx[4 * b + 3];
        const float4 p = l.dihd_p[b];                 // {k, cos(n v0), sin(n v0), n}
        const int nn = (int)p.w;
        const double4 rj = a.pos[i1], rk = a.pos[i2];
        const float3 r_ij = fdir(S, rj, a.pos[i0]);
        const float3 r_kj = fdir(S, rj, rk);
        const float3 r_lk = fdir(S, rk, a.pos[i3]);
        const float3 r_kl = make_float3(-r_lk.x, -r_lk.y, -r_lk.z);
        const float r_kj_lensq  = fdot(r_kj, r_kj);
        const float r_kj_rlen   = rsqrtf(r_kj_lensq);
        const float r_kj_len    = r_kj_rlen * r_kj_lensq;
        const float3 m = fcross(r_ij, r_kj);
        const float3 n = fcross(r_kj, r_kl);
        const float m_lensq = fdot(m, m);
        const float n_lensq = fdot(n, n);
        if(m_lensq < ILL_SIN * ILL_SIN * fdot(r_ij, r_ij) * r_kj_lensq ||
           n_lensq < ILL_SIN * ILL_SIN * fdot(r_kl, r_kl) * r_kj_lensq)
        {
            // a bond angle of the dihedral within 11.5 degrees of collinear:
            // the normals m, n lose their direction in FP32
            e = dihedral_fp64<PREC, NF, NE>(a, l, b, W);
        }
        else
        {
            // (cos phi, sin phi) of the reference's phi = copysign(acos(m.n), r_ij.n)
            const float x = fdot(m, n);
            const float y = r_kj_len * fdot(r_ij, n);
            const float h = rsqrtf(x * x + y * y);
            const float c1 = x * h, s1 = y * h;
            float cn = 1.0f, sn = 0.0f;
            const int na = nn < 0 ? -nn : nn;
            for(int q = 0; q < na; ++q)
            {
                const float c2 = cn * c1 - sn * s1;
                sn = sn * c1 + cn * s1;
                cn = c2;
            }
            if(nn < 0) {sn = -sn;}
            // cos, sin of n (phi - v0)
            const float cd = cn * p.y + sn * p.z;
            const float sd = sn * p.y - cn * p.z;
            if(NE) {e = (double)(p.x * (1.0f + cd));}
            if(NF)
            {
                const float coef = p.x * (float)nn * sd;     // -dV/dphi
                const float cfi =  coef * r_kj_len / m_lensq;
                const float cfl = -coef * r_kj_len / n_lensq;
                const float3 Fi = make_float3(cfi * m.x, cfi * m.y, cfi * m.z);
                const float3 Fl = make_float3(cfl * n.x, cfl * n.y, cfl * n.z);
                const float rl2 = r_kj_rlen * r_kj_rlen;
                const float cijk = fdot(r_ij, r_kj) * rl2;
                const float cjkl = fdot(r_kl, r_kj) * rl2;
                W.add(a.force, i0, Fi.x, Fi.y, Fi.z);
                W.add(a.force, i1, (cijk - 1.0f) * Fi.x - cjkl * Fl.x, (cijk - 1.0f) * Fi.y - cjkl * Fl.y,
                      (cijk - 1.0f) * Fi.z - cjkl * Fl.z);
                W.add(a.force, i2, (cjkl - 1.0f) * Fl.x - cijk * Fi.x, (cjkl - 1.0f) * Fl.y - cijk * Fi.y,
                      (cjkl - 1.0f) * Fl.z - cijk * Fi.z);
                W.add(a.force, i3, Fl.x, Fl.y, Fl.z);
            }
        }
    }
    if(NE) {reduce_energy(a, sys, active, e, T_DIHEDRAL);}
}

// One block per window of SEG particles: every bond, angle and dihedral whose
// smallest particle index falls in the window (terms are sorted by it at
// commit; win_* hold the per-window term ranges) adds its forces to the
// block's shared accumulator of SEG + HALO particles, which is flushed once
// per particle.  The trip counts are uniform over the block, so the warp
// energy reductions see whole warps.
// The mixed form is held to 48 registers (five blocks per SM): its FP64
// fallback for near-collinear geometry would otherwise set the register count
// (and the occupancy) of every thread; the rare fallback spills instead.
template<int PREC, bool NF, bool NE>
__global__ void __launch_bounds__(TPB, PREC == P_MIXED ? 5 : 3) k_local(Arena a, LocalArrays l, int mask)
{
    __shared__ typename WinT<PREC>::type win[3 * WINDOW];
    const int w = blockIdx.x;
    Window<PREC> W{win, w * SEG};
    if(NF)
    {
        for(int k = threadIdx.x; k < 3 * WINDOW; k += TPB) {win[k] = 0;}
        __syncthreads();
    }
    if(mask & 1)
    {
        const long long b0 = l.win_bond[w], b1 = l.win_bond[w + 1];
        for(long long base = b0; base < b1; base += TPB)
        {
            const long long b = base + threadIdx.x;
            if(PREC == P_FP64) {do_bond<PREC, NF, NE>(a, l, b, b < b1 && !(a.any_frozen && a.sys[l.bond_sys[b]].frozen), W);}
            else               {do_bond_f32<PREC, NF, NE>(a, l, b, b < b1 && !(a.any_frozen && a.sys[l.bond_sys[b]].frozen), W);}
        }
    }
    if(mask & 2)
    {
        const long long b0 = l.win_angle[w], b1 = l.win_angle[w + 1];
        for(long long base = b0; base < b1; base += TPB)
        {
            const long long b = base + threadIdx.x;
            if(PREC == P_FP64) {do_angle<PREC, NF, NE>(a, l, b, b < b1 && !(a.any_frozen && a.sys[l.angle_sys[b]].frozen), W);}
            else               {do_angle_f32<PREC, NF, NE>(a, l, b, b < b1 && !(a.any_frozen && a.sys[l.angle_sys[b]].frozen), W);}
        }
    }
    if(mask & 4)
    {
        const long long b0 = l.win_dihd[w], b1 = l.win_dihd[w + 1];
        for(long long base = b0; base < b1; base += TPB)
        {
            const long long b = base + threadIdx.x;
            if(PREC == P_FP64) {do_dihedral<PREC, NF, NE>(a, l, b, b < b1 && !(a.any_frozen && a.sys[l.dihd_sys[b]].frozen), W);}
            else               {do_dihedral_f32<PREC, NF, NE>(a, l, b, b < b1 && !(a.any_frozen && a.sys[l.dihd_sys[b]].frozen), W);}
        }
    }
    if(NF)
    {
        __syncthreads();
        W.flush(a.force, a.n);
    }
}

template<int PREC, bool NF, bool NE>
void run_all(const Arena& a, const LocalArrays& l, int mask, cudaStream_t s)
{
    if(l.nwin == 0 || (l.nbond + l.nangle + l.ndihd) == 0) {return;}
    k_local<PREC, NF, NE><<<l.nwin, TPB, 0, s>>>(a, l, mask);
    note_launches(1);
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
        // mixed form: forces in FP32 (the per-step path); energies, an
        // observable read between steps, in the reference's FP64 arithmetic
        if(nf)       {run_all<P_MIXED, true, false>(a, l, mask, s);}
        if(ne)       {run_all<P_FP64, false, true>(a, l, mask, s);}
    }
}

}  // namespace mjg
