// BAOAB Langevin and velocity-Verlet updates (core/BAOABLangevinIntegrator.hpp
// :170-240, core/VelocityVerletIntegrator.hpp:90-135), the Verlet-skin
// bookkeeping of reduce_margin (core/PeriodicGridCellList.hpp:100-110), and
// the host<->arena layout conversions.
//
// One thread per particle over every system of the arena; a particle finds its
// system's box, seed and step through psys.  Arithmetic is FP64 with explicit
// round-to-nearest products and sums, in the reference's operation order.
#include "kernels.cuh"

namespace mjg {

namespace {

constexpr int TPB = 256;

template<int PREC>
__device__ __forceinline__ void load_force(const void* force, long long i, double& fx, double& fy, double& fz)
{
    if(PREC == P_FP64)
    {
        const double4 f = static_cast<const double4*>(force)[i];
        fx = f.x; fy = f.y; fz = f.z;
    }
    else
    {
        const longlong4 f = static_cast<const longlong4*>(force)[i];
        fx = fx_to_double(f.x); fy = fx_to_double(f.y); fz = fx_to_double(f.z);
    }
}

template<int PREC>
__device__ __forceinline__ void zero_force(void* force, long long i)
{
    if(PREC == P_FP64) {static_cast<double4*>(force)[i] = make_double4(0, 0, 0, 0);}
    else               {static_cast<longlong4*>(force)[i] = make_longlong4(0, 0, 0, 0);}
}

// The closing half of an UnderdampedLangevin step
// (core/UnderdampedLangevinIntegrator.hpp:252-264): a = f/m + sigma R with the
// noise of counter `ctr`, v += halfdt (1 - gamma halfdt) a.
__device__ __forceinline__ void underdamped_close(const SysDev& S, long long i, double4& v, double4& acc,
                                                  const double4& c, double fx, double fy, double fz,
                                                  unsigned long long ctr)
{
    double r0, r1, r2;
    gaussian3(S.seed, (unsigned long long)(i - S.off), ctr, r0, r1, r2);
    acc.x = __dadd_rn(__dmul_rn(fx, c.x), __dmul_rn(r0, c.z));
    acc.y = __dadd_rn(__dmul_rn(fy, c.x), __dmul_rn(r1, c.z));
    acc.z = __dadd_rn(__dmul_rn(fz, c.x), __dmul_rn(r2, c.z));
    const double halfdt = c.w / 2;
    const double k = __dmul_rn(halfdt, __dsub_rn(1.0, __dmul_rn(c.y, halfdt)));
    v.x = __dadd_rn(v.x, __dmul_rn(k, acc.x));
    v.y = __dadd_rn(v.y, __dmul_rn(k, acc.y));
    v.z = __dadd_rn(v.z, __dmul_rn(k, acc.z));
}

// B-A-O-A of BAOAB (or the first half-kick and drift of velocity Verlet, or
// the first half of an UnderdampedLangevin or G-JF step), force reset and the
// per-system largest squared displacement.  With KICK the previous step's
// closing half is applied first, as separate rounding steps, so that
// consecutive steps of a chunk share one pass.  AUX: the arena holds
// UnderdampedLangevin or G-JF systems (their branches cost registers, and
// occupancy, in the BAOAB / velocity-Verlet arenas that have none).
template<int PREC, bool KICK, bool AUX>
__global__ void __launch_bounds__(TPB) k_integrate_first(Arena a)
{
    const long long i = (long long)blockIdx.x * TPB + threadIdx.x;
    const bool active = i < a.n;
    int s = active ? a.psys[i] : 0;
    double d2 = 0.0;
    if(active && !a.sys[s].frozen)
    {
        const SysDev& S = a.sys[s];
        double4 p = a.pos[i];
        double4 v = a.vel[i];
        const double4 c = S.uniform_coef ? S.coef : a.coef[i];     // per integrator: see Arena::coef
        double fx, fy, fz;
        load_force<PREC>(a.force, i, fx, fy, fz);
        const bool uld = AUX && S.integrator == I_UNDERDAMPED;
        if(KICK && !uld)
        {
            v.x = __dadd_rn(v.x, __dmul_rn(c.x, fx));
            v.y = __dadd_rn(v.y, __dmul_rn(c.x, fy));
            v.z = __dadd_rn(v.z, __dmul_rn(c.x, fz));
        }
        double dx, dy, dz;
        double4 pn = p;     // g-BAOAB: the new position, moved by its two half drifts
        bool direct = false;
        if(uld)             // core/UnderdampedLangevinIntegrator.hpp:198-221
        {
            double4 acc = a.accel[i];
            if(KICK) {underdamped_close(S, i, v, acc, c, fx, fy, fz, S.step); a.accel[i] = acc;}
            const double dt = c.w, halfdt = dt / 2, halfdt2 = dt * dt / 2;
            const double gdo2 = __dmul_rn(c.y, halfdt);                 // gamma dt / 2
            const double omg  = __dsub_rn(1.0, gdo2);
            const double cv   = __dmul_rn(dt, omg);
            dx = __dadd_rn(__dmul_rn(cv, v.x), __dmul_rn(halfdt2, acc.x));
            dy = __dadd_rn(__dmul_rn(cv, v.y), __dmul_rn(halfdt2, acc.y));
            dz = __dadd_rn(__dmul_rn(cv, v.z), __dmul_rn(halfdt2, acc.z));
            const double sv = __dmul_rn(omg, __dadd_rn(__dmul_rn(omg, omg), gdo2));
            v.x = __dmul_rn(v.x, sv);
            v.y = __dmul_rn(v.y, sv);
            v.z = __dmul_rn(v.z, sv);
            const double sa = __dmul_rn(halfdt, omg);
            v.x = __dadd_rn(v.x, __dmul_rn(sa, acc.x));
            v.y = __dadd_rn(v.y, __dmul_rn(sa, acc.y));
            v.z = __dadd_rn(v.z, __dmul_rn(sa, acc.z));
        }
        else if(AUX && S.integrator == I_GJF)   // core/GJFNVTLangevinIntegrator.hpp:183-204
        {
            double r0, r1, r2;
            gaussian3(S.seed, (unsigned long long)(i - S.off), S.step, r0, r1, r2);
            const double4 x = a.accel[i];                       // {1/2m, b/m, b dt}
            const double b0 = __dmul_rn(r0, c.z), b1 = __dmul_rn(r1, c.z), b2 = __dmul_rn(r2, c.z);
            // dp = (b dt) (v + 1/2m (dt f + beta))
            dx = __dmul_rn(x.z, __dadd_rn(v.x, __dmul_rn(x.x, __dadd_rn(__dmul_rn(c.w, fx), b0))));
            dy = __dmul_rn(x.z, __dadd_rn(v.y, __dmul_rn(x.x, __dadd_rn(__dmul_rn(c.w, fy), b1))));
            dz = __dmul_rn(x.z, __dadd_rn(v.z, __dmul_rn(x.x, __dadd_rn(__dmul_rn(c.w, fz), b2))));
            // v = a (v + (dt/2m) f) + (b/m) beta
            v.x = __dadd_rn(__dmul_rn(c.y, __dadd_rn(v.x, __dmul_rn(c.x, fx))), __dmul_rn(x.y, b0));
            v.y = __dadd_rn(__dmul_rn(c.y, __dadd_rn(v.y, __dmul_rn(c.x, fy))), __dmul_rn(x.y, b1));
            v.z = __dadd_rn(__dmul_rn(c.y, __dadd_rn(v.z, __dmul_rn(c.x, fz))), __dmul_rn(x.y, b2));
        }
        else if(S.integrator == I_BAOAB || S.integrator == I_GBAOAB)
        {
            // g-BAOAB without constraints (gBAOABLangevinIntegrator.hpp:318-420,
            // one correction step): the same B-A-O-A, but each half drift moves
            // the position itself and the displacement is new minus old position
            const bool split = S.integrator == I_GBAOAB;
            double r0, r1, r2;
            gaussian3(S.seed, (unsigned long long)(i - S.off), S.step, r0, r1, r2);
            v.x = __dadd_rn(v.x, __dmul_rn(c.x, fx));          // v += halfdt*rm*f
            v.y = __dadd_rn(v.y, __dmul_rn(c.x, fy));
            v.z = __dadd_rn(v.z, __dmul_rn(c.x, fz));
            dx = __dmul_rn(c.w, v.x);                          // dp  = halfdt*v
            dy = __dmul_rn(c.w, v.y);
            dz = __dmul_rn(c.w, v.z);
            if(split) {pn = make_double4(__dadd_rn(p.x, dx), __dadd_rn(p.y, dy), __dadd_rn(p.z, dz), p.w);}
            v.x = __dmul_rn(v.x, c.y);                         // v  *= exp(-gamma dt)
            v.y = __dmul_rn(v.y, c.y);
            v.z = __dmul_rn(v.z, c.y);
            v.x = __dadd_rn(v.x, __dmul_rn(c.z, r0));          // v  += noise*R
            v.y = __dadd_rn(v.y, __dmul_rn(c.z, r1));
            v.z = __dadd_rn(v.z, __dmul_rn(c.z, r2));
            if(split)
            {
                pn.x = __dadd_rn(pn.x, __dmul_rn(c.w, v.x));
                pn.y = __dadd_rn(pn.y, __dmul_rn(c.w, v.y));
                pn.z = __dadd_rn(pn.z, __dmul_rn(c.w, v.z));
                dx = __dsub_rn(pn.x, p.x);                     // displacement = new - old
                dy = __dsub_rn(pn.y, p.y);
                dz = __dsub_rn(pn.z, p.z);
                direct = true;
            }
            else
            {
                dx = __dadd_rn(dx, __dmul_rn(c.w, v.x));       // dp += halfdt*v
                dy = __dadd_rn(dy, __dmul_rn(c.w, v.y));
                dz = __dadd_rn(dz, __dmul_rn(c.w, v.z));
            }
        }
        else
        {
            v.x = __dadd_rn(v.x, __dmul_rn(c.x, fx));          // v += (halfdt*rm)*f
            v.y = __dadd_rn(v.y, __dmul_rn(c.x, fy));
            v.z = __dadd_rn(v.z, __dmul_rn(c.x, fz));
            dx = __dmul_rn(c.w, v.x);                          // disp = dt*v
            dy = __dmul_rn(c.w, v.y);
            dz = __dmul_rn(c.w, v.z);
        }
        if(direct) {p = pn;}
        else
        {
            p.x = __dadd_rn(p.x, dx);
            p.y = __dadd_rn(p.y, dy);
            p.z = __dadd_rn(p.z, dz);
        }
        if(S.boundary == B_PERIODIC)                           // adjust_position
        {
            if(p.x < S.lower[0]) {p.x = __dadd_rn(p.x, S.width[0]);} else if(p.x >= S.upper[0]) {p.x = __dsub_rn(p.x, S.width[0]);}
            if(p.y < S.lower[1]) {p.y = __dadd_rn(p.y, S.width[1]);} else if(p.y >= S.upper[1]) {p.y = __dsub_rn(p.y, S.width[1]);}
            if(p.z < S.lower[2]) {p.z = __dadd_rn(p.z, S.width[2]);} else if(p.z >= S.upper[2]) {p.z = __dsub_rn(p.z, S.width[2]);}
        }
        a.pos[i] = p;
        a.vel[i] = v;
        // the pair kernels read coordinates in slot order: keep every term's
        // copy current (a rebuild later in the step renumbers its systems'
        // slots and rewrites them)
#pragma unroll
        for(int g = 0; g < NGLOBAL; ++g)
        {
            if(a.slot_of[g])
            {
                const int so = a.slot_of[g][i];
                if(so >= 0) {a.slot_pd[g][so] = make_double4(p.x, p.y, p.z, a.slot_w[g][i]);}   // whole 32 B
            }
        }
        zero_force<PREC>(a.force, i);
        d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
        if(!(d2 == d2) || d2 > 1e300) {atomicOr(&a.sys[s].status, ST_NONFINITE); d2 = 0.0;}
    }
    // per-system maximum: warp-level when the warp sits in one system
    const unsigned full = 0xffffffffu;
    const int s0 = __shfl_sync(full, s, 0);
    const bool uniform = __all_sync(full, !active || s == s0);
    if(uniform)
    {
        double m = d2;
#pragma unroll
        for(int o = 16; o > 0; o >>= 1) {m = fmax(m, __shfl_xor_sync(full, m, o));}
        const bool any = __any_sync(full, active);
        if(any && (threadIdx.x & 31) == 0)
        {
            atomicMax(&a.sys[s0].max_disp2, (unsigned long long)__double_as_longlong(m));
        }
    }
    else if(active)
    {
        atomicMax(&a.sys[s].max_disp2, (unsigned long long)__double_as_longlong(d2));
    }
}

// reduce_margin(2 sqrt(max|dp|^2)) for every global term of every system;
// a term whose skin is used up is flagged for a rebuild.  Also advances the
// noise step counter.
__global__ void k_margin(Arena a, int* any0, int* any1, int* any2, RebuildGate gate)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if(s >= a.nsys) {return;}
    SysDev& S = a.sys[s];
    if(S.frozen) {return;}
    const double d = 2 * sqrt(__longlong_as_double((long long)S.max_disp2));
    S.max_disp2 = 0ull;
    S.step += 1ull;
    int* any[3] = {any0, any1, any2};
    for(int g = 0; g < NGLOBAL; ++g)
    {
        GlobalParams& G = S.g[g];
        if(!G.on) {continue;}
        G.current_margin = __dsub_rn(G.current_margin, d);
        if(G.current_margin < 0)
        {
            G.rebuild = 1;
            if(any[g]) {atomicOr(any[g], 1);}
            if(gate.on[g]) {cudaGraphSetConditional(gate.handle[g], 1u);}   // the term's rebuild runs
        }
    }
}

// closing half of the last step of a chunk: v += (halfdt/m) f (BAOAB,
// velocity Verlet, G-JF) or the UnderdampedLangevin closing
template<int PREC>
__global__ void __launch_bounds__(TPB) k_integrate_last(Arena a)
{
    const long long i = (long long)blockIdx.x * TPB + threadIdx.x;
    if(i >= a.n) {return;}
    const SysDev& S = a.sys[a.psys[i]];
    if(S.frozen) {return;}
    double fx, fy, fz;
    load_force<PREC>(a.force, i, fx, fy, fz);
    double4 v = a.vel[i];
    if(S.integrator == I_UNDERDAMPED)
    {
        double4 acc = a.accel[i];
        underdamped_close(S, i, v, acc, S.uniform_coef ? S.coef : a.coef[i], fx, fy, fz, S.step);
        a.accel[i] = acc;
        a.vel[i] = v;
        return;
    }
    const double c = S.uniform_coef ? S.coef.x : a.coef[i].x;
    v.x = __dadd_rn(v.x, __dmul_rn(c, fx));
    v.y = __dadd_rn(v.y, __dmul_rn(c, fy));
    v.z = __dadd_rn(v.z, __dmul_rn(c, fz));
    a.vel[i] = v;
}

// UnderdampedLangevinIntegrator::initialize (:160-181): a = f/m + sigma R,
// with the noise counter at the system's current step (a resumed system gets
// the acceleration the uninterrupted run had)
template<int PREC>
__global__ void k_init_accel(Arena a, long long first, long long count)
{
    const long long k = (long long)blockIdx.x * TPB + threadIdx.x;
    if(k >= count) {return;}
    const long long i = first + k;
    const SysDev& S = a.sys[a.psys[i]];
    if(S.integrator != I_UNDERDAMPED) {return;}
    double fx, fy, fz;
    load_force<PREC>(a.force, i, fx, fy, fz);
    const double4 c = S.uniform_coef ? S.coef : a.coef[i];
    double r0, r1, r2;
    gaussian3(S.seed, (unsigned long long)(i - S.off), S.step, r0, r1, r2);
    a.accel[i] = make_double4(__dadd_rn(__dmul_rn(fx, c.x), __dmul_rn(r0, c.z)),
                              __dadd_rn(__dmul_rn(fy, c.x), __dmul_rn(r1, c.z)),
                              __dadd_rn(__dmul_rn(fz, c.x), __dmul_rn(r2, c.z)), 0.0);
}

template<int PREC>
__global__ void k_zero_force(Arena a)
{
    const long long i = (long long)blockIdx.x * TPB + threadIdx.x;
    if(i < a.n && !a.sys[a.psys[i]].frozen) {zero_force<PREC>(a.force, i);}
}

__global__ void k_unpack(Arena a, const double* src_pos, const double* src_vel, long long first, long long count)
{
    const long long k = (long long)blockIdx.x * TPB + threadIdx.x;
    if(k >= count) {return;}
    const long long i = first + k;
    if(src_pos) {a.pos[i] = make_double4(src_pos[3*k], src_pos[3*k+1], src_pos[3*k+2], 0.0);}
    if(src_vel) {a.vel[i] = make_double4(src_vel[3*k], src_vel[3*k+1], src_vel[3*k+2], 0.0);}
}

template<int PREC>
__global__ void k_pack(Arena a, double* dst, int what, long long first, long long count)
{
    const long long k = (long long)blockIdx.x * TPB + threadIdx.x;
    if(k >= count) {return;}
    const long long i = first + k;
    double x, y, z;
    if(what == 0)      {const double4 p = a.pos[i]; x = p.x; y = p.y; z = p.z;}
    else if(what == 1) {const double4 v = a.vel[i]; x = v.x; y = v.y; z = v.z;}
    else if(what == 3) {const double4 q = a.accel ? a.accel[i] : make_double4(0, 0, 0, 0); x = q.x; y = q.y; z = q.z;}
    else               {load_force<PREC>(a.force, i, x, y, z);}
    dst[3*k] = x; dst[3*k+1] = y; dst[3*k+2] = z;
}

template<int PREC>
__global__ void k_set_force(Arena a, const double* src, long long first, long long count)
{
    const long long k = (long long)blockIdx.x * TPB + threadIdx.x;
    if(k >= count) {return;}
    const long long i = first + k;
    if(PREC == P_FP64)
    {
        static_cast<double4*>(a.force)[i] = make_double4(src[3*k], src[3*k+1], src[3*k+2], 0.0);
    }
    else
    {
        static_cast<longlong4*>(a.force)[i] = make_longlong4(fx_from_double(src[3*k]),
            fx_from_double(src[3*k+1]), fx_from_double(src[3*k+2]), 0);
    }
}

__global__ void k_set_noise(Arena a, const double* src, long long first, long long count)
{
    const long long k = (long long)blockIdx.x * TPB + threadIdx.x;
    if(k < count) {a.coef[first + k].z = src[k];}
}

__global__ void k_clear_energy(Arena a)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if(s >= a.nsys) {return;}
    for(int t = 0; t < NTERMS; ++t) {a.sys[s].energy[t] = 0.0;}
}

inline unsigned blocks(long long n) {return (unsigned)((n + TPB - 1) / TPB);}

}  // namespace

void launch_integrate_first(const Arena& a, cudaStream_t s, bool kick)
{
    if(a.n == 0) {return;}
    const bool aux = a.accel != nullptr;
    const int nb = (int)blocks(a.n);
    if(a.precision == P_FP64)
    {
        if(aux) {if(kick) {k_integrate_first<P_FP64, true,  true ><<<nb, TPB, 0, s>>>(a);}
                 else     {k_integrate_first<P_FP64, false, true ><<<nb, TPB, 0, s>>>(a);}}
        else    {if(kick) {k_integrate_first<P_FP64, true,  false><<<nb, TPB, 0, s>>>(a);}
                 else     {k_integrate_first<P_FP64, false, false><<<nb, TPB, 0, s>>>(a);}}
    }
    else
    {
        if(aux) {if(kick) {k_integrate_first<P_MIXED, true,  true ><<<nb, TPB, 0, s>>>(a);}
                 else     {k_integrate_first<P_MIXED, false, true ><<<nb, TPB, 0, s>>>(a);}}
        else    {if(kick) {k_integrate_first<P_MIXED, true,  false><<<nb, TPB, 0, s>>>(a);}
                 else     {k_integrate_first<P_MIXED, false, false><<<nb, TPB, 0, s>>>(a);}}
    }
    note_launches(1);
}

void launch_margin(const Arena& a, TermArrays* t, cudaStream_t s, const RebuildGate& gate)
{
    if(a.nsys == 0) {return;}
    k_margin<<<(a.nsys + 127) / 128, 128, 0, s>>>(a,
        t[0].on ? t[0].any_rebuild : nullptr, t[1].on ? t[1].any_rebuild : nullptr,
        t[2].on ? t[2].any_rebuild : nullptr, gate);
    note_launches(1);
}

__global__ void k_set_accel(Arena a, const double* src, long long first, long long count)
{
    const long long k = (long long)blockIdx.x * TPB + threadIdx.x;
    if(k < count) {a.accel[first + k] = make_double4(src[3 * k], src[3 * k + 1], src[3 * k + 2], 0.0);}
}

void launch_set_accel(const Arena& a, const double* src, long long first, long long count, cudaStream_t s)
{
    if(count == 0 || !a.accel) {return;}
    k_set_accel<<<blocks(count), TPB, 0, s>>>(a, src, first, count);
    note_launches(1);
}

void launch_init_accel(const Arena& a, long long first, long long count, cudaStream_t s)
{
    if(count == 0 || !a.accel) {return;}
    if(a.precision == P_FP64) {k_init_accel<P_FP64><<<blocks(count), TPB, 0, s>>>(a, first, count);}
    else                      {k_init_accel<P_MIXED><<<blocks(count), TPB, 0, s>>>(a, first, count);}
    note_launches(1);
}

void launch_integrate_last(const Arena& a, cudaStream_t s)
{
    if(a.n == 0) {return;}
    if(a.precision == P_FP64) {k_integrate_last<P_FP64><<<blocks(a.n), TPB, 0, s>>>(a);}
    else                      {k_integrate_last<P_MIXED><<<blocks(a.n), TPB, 0, s>>>(a);}
    note_launches(1);
}

void launch_zero_force(const Arena& a, cudaStream_t s)
{
    if(a.n == 0) {return;}
    if(a.precision == P_FP64) {k_zero_force<P_FP64><<<blocks(a.n), TPB, 0, s>>>(a);}
    else                      {k_zero_force<P_MIXED><<<blocks(a.n), TPB, 0, s>>>(a);}
    note_launches(1);
}

void launch_unpack_state(const Arena& a, const double* src_pos, const double* src_vel,
                         long long first, long long count, cudaStream_t s)
{
    if(count == 0) {return;}
    k_unpack<<<blocks(count), TPB, 0, s>>>(a, src_pos, src_vel, first, count);
    note_launches(1);
}

void launch_pack_state(const Arena& a, double* dst, int what, long long first, long long count,
                       cudaStream_t s)
{
    if(count == 0) {return;}
    if(a.precision == P_FP64) {k_pack<P_FP64><<<blocks(count), TPB, 0, s>>>(a, dst, what, first, count);}
    else                      {k_pack<P_MIXED><<<blocks(count), TPB, 0, s>>>(a, dst, what, first, count);}
    note_launches(1);
}

void launch_clear_energy(const Arena& a, cudaStream_t s)
{
    if(a.nsys == 0) {return;}
    k_clear_energy<<<(a.nsys + 127) / 128, 128, 0, s>>>(a);
    note_launches(1);
}

// reads `n` int4 words and keeps one word of the result (only when it takes
// an impossible value), so that every line read stays clean in L2
__global__ void k_read_sweep(const int4* __restrict__ p, long long n, int* sink)
{
    int acc = 0;
    for(long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
        k += (long long)gridDim.x * blockDim.x)
    {
        const int4 w = __ldcg(p + k);
        acc ^= w.x ^ w.y ^ w.z ^ w.w;
    }
    if(acc == 0x7fffffff && sink) {*sink = acc;}
}

void launch_read_sweep(const void* p, size_t bytes, int* sink, cudaStream_t s)
{
    const long long n = (long long)(bytes / sizeof(int4));
    if(n == 0) {return;}
    k_read_sweep<<<148 * 8, 256, 0, s>>>(static_cast<const int4*>(p), n, sink);
    note_launches(1);
}

void launch_set_noise(const Arena& a, const double* noise, long long first, long long count,
                      cudaStream_t s)
{
    if(count == 0) {return;}
    k_set_noise<<<blocks(count), TPB, 0, s>>>(a, noise, first, count);
    note_launches(1);
}

void launch_set_force(const Arena& a, const double* src, long long first, long long count,
                      cudaStream_t s)
{
    if(count == 0) {return;}
    if(a.precision == P_FP64) {k_set_force<P_FP64><<<blocks(count), TPB, 0, s>>>(a, src, first, count);}
    else                      {k_set_force<P_MIXED><<<blocks(count), TPB, 0, s>>>(a, src, first, count);}
    note_launches(1);
}

}  // namespace mjg
