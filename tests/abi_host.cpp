// A C++ host of the C ABI, the way an application binds the library without
// Python: it reads one system from a flat binary file, builds it through
// include/mjolnir_b200.h (particles, harmonic bonds, angles, cosine
// dihedrals, ExcludedVolume and DebyeHuckel with particles_within.bond
// exclusions, BAOAB), advances it and writes the final positions,
// velocities, forces and per-term energies.
//
//   abi_host <in.bin> <out.bin> <precision: 0 fp64 | 1 mixed> <steps>
//
// Input layout (little endian, int64 counts, float64 reals unless noted):
//   n, pos[3n], vel[3n], mass[n], temperature, ionic_strength, dt, seed (uint64), gamma[n],
//   nb, bond_idx[2nb] (int64), bond_k[nb], bond_v0[nb],
//   na, angle_idx[3na], angle_k[na], angle_v0[na],
//   nd, dihd_idx[4nd], dihd_k[nd], dihd_n[nd] (int32), dihd_v0[nd],
//   nx, exv_idx[nx], exv_radius[nx], exv_eps, exv_cutoff, exv_margin,
//   nq, dh_idx[nq], dh_charge[nq], dh_cutoff, dh_margin, within_bond (int32)
// Output: pos[3n], vel[3n], force[3n], energies[6].
#include "mjolnir_b200.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

namespace {

struct Reader {
    std::FILE* f;
    template<typename T> T one()
    {
        T v{};
        if(std::fread(&v, sizeof(T), 1, f) != 1) {std::fprintf(stderr, "short input\n"); std::exit(2);}
        return v;
    }
    template<typename T> std::vector<T> many(int64_t k)
    {
        std::vector<T> v((size_t)k);
        if(k > 0 && std::fread(v.data(), sizeof(T), (size_t)k, f) != (size_t)k)
        {
            std::fprintf(stderr, "short input\n");
            std::exit(2);
        }
        return v;
    }
};

void check(mjg_context* ctx, int code, const char* what)
{
    if(code != MJG_OK)
    {
        std::fprintf(stderr, "%s failed (%d): %s\n", what, code, ctx ? mjg_last_error(ctx) : "");
        std::exit(1);
    }
}

}  // namespace

int main(int argc, char** argv)
{
    if(argc != 5) {std::fprintf(stderr, "usage: abi_host in.bin out.bin precision steps\n"); return 2;}
    std::FILE* in = std::fopen(argv[1], "rb");
    if(!in) {std::perror(argv[1]); return 2;}
    Reader r{in};
    const int64_t n = r.one<int64_t>();
    const auto pos = r.many<double>(3 * n), vel = r.many<double>(3 * n), mass = r.many<double>(n);
    const double T = r.one<double>(), I = r.one<double>(), dt = r.one<double>();
    const uint64_t seed = r.one<uint64_t>();
    const auto gamma = r.many<double>(n);
    const int64_t nb = r.one<int64_t>();
    const auto b_idx = r.many<int64_t>(2 * nb);
    const auto b_k = r.many<double>(nb), b_v0 = r.many<double>(nb);
    const int64_t na = r.one<int64_t>();
    const auto a_idx = r.many<int64_t>(3 * na);
    const auto a_k = r.many<double>(na), a_v0 = r.many<double>(na);
    const int64_t nd = r.one<int64_t>();
    const auto d_idx = r.many<int64_t>(4 * nd);
    const auto d_k = r.many<double>(nd);
    const auto d_n = r.many<int32_t>(nd);
    const auto d_v0 = r.many<double>(nd);
    const int64_t nx = r.one<int64_t>();
    const auto x_idx = r.many<int64_t>(nx);
    const auto x_r = r.many<double>(nx);
    const double x_eps = r.one<double>(), x_cut = r.one<double>(), x_margin = r.one<double>();
    const int64_t nq = r.one<int64_t>();
    const auto q_idx = r.many<int64_t>(nq);
    const auto q_c = r.many<double>(nq);
    const double q_cut = r.one<double>(), q_margin = r.one<double>();
    const int32_t within = r.one<int32_t>();
    std::fclose(in);

    mjg_context* ctx = nullptr;
    check(nullptr, mjg_context_create(0, std::atoi(argv[3]) ? MJG_PRECISION_MIXED : MJG_PRECISION_FP64, &ctx),
          "mjg_context_create");
    int sys = -1;
    const double zero[3] = {0.0, 0.0, 0.0};
    check(ctx, mjg_system_create(ctx, n, MJG_UNLIMITED, zero, zero, pos.data(), vel.data(), mass.data(), &sys),
          "mjg_system_create");
    check(ctx, mjg_system_set_attributes(ctx, sys, T, I), "mjg_system_set_attributes");
    check(ctx, mjg_bonds_set(ctx, sys, "bond", nb, b_idx.data(), b_k.data(), b_v0.data()), "mjg_bonds_set");
    check(ctx, mjg_angles_set(ctx, sys, "none", na, a_idx.data(), a_k.data(), a_v0.data()), "mjg_angles_set");
    check(ctx, mjg_dihedrals_set(ctx, sys, "none", nd, d_idx.data(), d_k.data(), d_n.data(), d_v0.data()),
          "mjg_dihedrals_set");
    check(ctx, mjg_exv_set(ctx, sys, x_eps, x_cut, x_margin, nx, x_idx.data(), x_r.data()), "mjg_exv_set");
    check(ctx, mjg_dh_set(ctx, sys, q_cut, q_margin, nq, q_idx.data(), q_c.data()), "mjg_dh_set");
    const char* kinds[1] = {"bond"};
    for(int term : {MJG_TERM_EXV, MJG_TERM_DH})
    {
        check(ctx, mjg_ignore_set(ctx, sys, term, MJG_IGNORE_NOTHING, within > 0 ? 1 : 0, kinds, &within),
              "mjg_ignore_set");
    }
    check(ctx, mjg_integrator_set(ctx, sys, MJG_BAOAB, dt, gamma.data(), seed), "mjg_integrator_set");
    check(ctx, mjg_commit(ctx), "mjg_commit");
    check(ctx, mjg_step(ctx, std::atoll(argv[4])), "mjg_step");

    std::vector<double> p(3 * n), v(3 * n), f(3 * n), e(6);
    check(ctx, mjg_get_state(ctx, sys, p.data(), v.data(), f.data()), "mjg_get_state");
    check(ctx, mjg_energies(ctx, sys, e.data()), "mjg_energies");
    mjg_context_destroy(ctx);

    std::FILE* out = std::fopen(argv[2], "wb");
    if(!out) {std::perror(argv[2]); return 2;}
    std::fwrite(p.data(), sizeof(double), p.size(), out);
    std::fwrite(v.data(), sizeof(double), v.size(), out);
    std::fwrite(f.data(), sizeof(double), f.size(), out);
    std::fwrite(e.data(), sizeof(double), e.size(), out);
    std::fclose(out);
    return 0;
}
