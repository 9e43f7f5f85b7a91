// TEST INFRASTRUCTURE ONLY -- not part of the product path.
//
// Runs one system, built by the reference's own code, either through the
// reference's MolecularDynamicsSimulator (core/MolecularDynamicsSimulator.hpp
// :13-125) on the CPU or through B200Simulator (B200Simulator.hpp, the
// reference-side binding of the C ABI) on the GPU, both behind SimulatorBase:
// initialize(), step() until it returns false, finalize().  The System and
// the ForceField come from oracle/ref_driver.cpp's RefSim, which assembles the
// reference's objects the way its input readers do.  Built by
// tests/binding/Makefile into tests/binding/_build/libb200_binding.so, linked
// against the product library.

#include "ref_driver.cpp"

#include <mjolnir/core/MolecularDynamicsSimulator.hpp>
#include <mjolnir/core/ObserverContainer.hpp>
#include <mjolnir/core/EnergyObserver.hpp>

#include "B200Simulator.hpp"

namespace
{

template<typename traitsT>
void copy_state(const System<traitsT>& sys, double* pos, double* vel)
{
    for(std::size_t i = 0; i < sys.size(); ++i)
    {
        const auto& r = sys.position(i);
        const auto& v = sys.velocity(i);
        pos[3 * i] = math::X(r); pos[3 * i + 1] = math::Y(r); pos[3 * i + 2] = math::Z(r);
        vel[3 * i] = math::X(v); vel[3 * i + 1] = math::Y(v); vel[3 * i + 2] = math::Z(v);
    }
}

template<typename traitsT>
double kinetic(const System<traitsT>& sys)
{
    double k = 0.0;
    for(std::size_t i = 0; i < sys.size(); ++i)
    {
        const auto& v = sys.velocity(i);
        k += 0.5 * sys.mass(i) * (math::X(v) * math::X(v) + math::Y(v) * math::Y(v) + math::Z(v) * math::Z(v));
    }
    return k;
}

// where: 0 = the reference's MolecularDynamicsSimulator (CPU), 1 =
// B200Simulator (GPU).  energy[0] = potential + kinetic energy after the run.
template<typename traitsT>
void run_impl(const orc_spec& s, int where, int precision, long long steps, const char* prefix,
              double* pos, double* vel, double* energy)
{
    using vv_type = VelocityVerletIntegrator<traitsT>;
    RefSim<traitsT, true> built(s);           // the reference's System and ForceField
    vv_type integr(s.dt, SystemMotionRemover<traitsT>(false, false, false));
    if(where == 0)
    {
        ObserverContainer<traitsT> obs(false);
        obs.push_back(make_unique<EnergyObserver<traitsT>>(std::string(prefix)));
        MolecularDynamicsSimulator<traitsT, vv_type> sim(std::size_t(steps), std::size_t(steps),
            std::size_t(steps), std::move(*built.sys), std::move(built.ff), std::move(integr), std::move(obs),
            RandomNumberGenerator<traitsT>(static_cast<std::uint32_t>(s.seed)));
        SimulatorBase& base = sim;
        base.initialize();
        while(base.step()) {}
        base.finalize();
        copy_state(sim.system(), pos, vel);
        *energy = sim.forcefields()->calc_energy(sim.system()) + kinetic(sim.system());
    }
    else
    {
        B200IgnoreRule ignore;
        ignore.molecule = s.ignore_molecule == ORC_IGNORE_SELF   ? "Self"   :
                          s.ignore_molecule == ORC_IGNORE_OTHERS ? "Others" : "Nothing";
        if(s.ignore_bond_within > 0) {ignore.within["bond"] = std::size_t(s.ignore_bond_within);}
        std::map<std::string, B200PairInput> inputs;
        if(s.exv_on)
        {
            B200PairInput& in = inputs["ExcludedVolume"];
            for(long long k = 0; k < s.exv_n; ++k)
            {
                in.participants.push_back(std::size_t(s.exv_idx[k]));
                in.p0.push_back(s.exv_radius[k]);
            }
        }
        if(s.dh_on)
        {
            B200PairInput& in = inputs["DebyeHuckel"];
            for(long long k = 0; k < s.dh_n; ++k)
            {
                in.participants.push_back(std::size_t(s.dh_idx[k]));
                in.p0.push_back(s.dh_charge[k]);
            }
        }
        if(s.lj_on)
        {
            B200PairInput& in = inputs["LennardJones"];
            for(long long k = 0; k < s.lj_n; ++k)
            {
                in.participants.push_back(std::size_t(s.lj_idx[k]));
                in.p0.push_back(s.lj_sigma[k]);
                in.p1.push_back(s.lj_eps[k]);
            }
        }
        B200Simulator<traitsT, vv_type> sim(std::size_t(steps), std::move(*built.sys), std::move(built.ff),
                                            std::move(integr), ignore, std::move(inputs), precision);
        SimulatorBase& base = sim;
        base.initialize();
        while(base.step()) {}
        base.finalize();
        copy_state(sim.system(), pos, vel);
        *energy = sim.calc_energy() + kinetic(sim.system());
    }
}

} // anonymous

extern "C" {

// Returns 0, or -1 with the message in bind_last_error().
int bind_run(const orc_spec* s, int where, int precision, long long steps, const char* prefix,
             double* pos, double* vel, double* energy)
{
    try
    {
        set_units_once();
        if(s->boundary == 1)
        {
            run_impl<SimulatorTraits<double, CuboidalPeriodicBoundary>>(*s, where, precision, steps, prefix,
                                                                       pos, vel, energy);
        }
        else
        {
            run_impl<SimulatorTraits<double, UnlimitedBoundary>>(*s, where, precision, steps, prefix,
                                                                pos, vel, energy);
        }
        return 0;
    }
    catch(const std::exception& e)
    {
        g_error = e.what();
        return -1;
    }
}

const char* bind_last_error() {return g_error.c_str();}

} // extern "C"
