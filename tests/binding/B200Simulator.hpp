// B200Simulator: the reference-side binding of the B200 hot path.
//
// This header is what a Mjolnir maintainer adds to the reference tree (as
// mjolnir/gpu/B200Simulator.hpp) to run a simulation's per-step hot path on a
// B200 behind the reference's own simulator interface: it derives from
// SimulatorBase (core/SimulatorBase.hpp:7-16), takes the System, the ForceField
// and the integrator the reference's input readers build
// (input/read_simulator.hpp:418-530), reads every supported interaction's
// parameters through the reference's public accessors, and drives the C ABI of
// include/mjolnir_b200.h.  It replaces MolecularDynamicsSimulator<traitsT,
// integratorT> (core/MolecularDynamicsSimulator.hpp:13-125) for systems made of
//   BondLengthInteraction<Harmonic>, BondAngleInteraction<Harmonic>,
//   DihedralAngleInteraction<Cosine>, DummyInteraction (topology only),
//   GlobalPairInteraction<ExcludedVolume / DebyeHuckel / LennardJones>,
// with a VelocityVerletIntegrator or a BAOABLangevinIntegrator, in either
// boundary.  Anything else throws std::runtime_error from the constructor,
// like the reference's readers.
//
// Two things the reference's objects keep private come from the reader that
// builds this simulator, as it hands them to the reference's own objects: the
// [[forcefields.global]] ignore table (molecule rule and connection distances,
// private in ExclusionList) and the participants of each pair interaction with
// their per-particle parameters (the specialised ExcludedVolume and
// LennardJones interactions have no parameters() accessor, and the generic
// GlobalPairInteraction's const one, GlobalPairInteraction.hpp:115, does not
// compile: it returns the list's base class as the list).  The system's state lives on the GPU between initialize() and
// finalize(); finalize() writes positions, velocities and forces back into the
// reference System, which system() returns.
//
// Built against the reference headers by tests/binding/Makefile for the test
// tests/test_gpu_binding.py.
#ifndef MJOLNIR_B200_SIMULATOR_HPP
#define MJOLNIR_B200_SIMULATOR_HPP
#include <mjolnir/core/SimulatorBase.hpp>
#include <mjolnir/core/System.hpp>
#include <mjolnir/core/ForceField.hpp>
#include <mjolnir/core/BoundaryCondition.hpp>
#include <mjolnir/core/VelocityVerletIntegrator.hpp>
#include <mjolnir/core/BAOABLangevinIntegrator.hpp>
#include <mjolnir/forcefield/global/GlobalPairInteraction.hpp>
#include <mjolnir/forcefield/global/GlobalPairExcludedVolumeInteraction.hpp>
#include <mjolnir/forcefield/global/GlobalPairLennardJonesInteraction.hpp>
#include <mjolnir/forcefield/global/ExcludedVolumePotential.hpp>
#include <mjolnir/forcefield/global/DebyeHuckelPotential.hpp>
#include <mjolnir/forcefield/global/LennardJonesPotential.hpp>
#include <mjolnir/forcefield/local/BondLengthInteraction.hpp>
#include <mjolnir/forcefield/local/BondAngleInteraction.hpp>
#include <mjolnir/forcefield/local/DihedralAngleInteraction.hpp>
#include <mjolnir/forcefield/local/DummyInteraction.hpp>
#include <mjolnir/forcefield/local/HarmonicPotential.hpp>
#include <mjolnir/forcefield/local/CosinePotential.hpp>
#include <mjolnir_b200.h>

#include <algorithm>
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

namespace mjolnir
{

// the [[forcefields.global]] ignore table of one pair interaction
struct B200IgnoreRule
{
    std::string molecule = "Nothing";                  // "Nothing" | "Self" | "Others"
    std::map<std::string, std::size_t> within;         // connection kind -> distance
};

// the participants of an ExcludedVolume (p0 = radius), DebyeHuckel (p0 =
// charge) or LennardJones (p0 = sigma, p1 = epsilon) interaction, as the
// reader parsed them
struct B200PairInput
{
    std::vector<std::size_t> participants;
    std::vector<double> p0, p1;
};

template<typename traitsT, typename integratorT>
class B200Simulator final : public SimulatorBase
{
  public:
    using traits_type     = traitsT;
    using real_type       = typename traits_type::real_type;
    using coordinate_type = typename traits_type::coordinate_type;
    using boundary_type   = typename traits_type::boundary_type;
    using system_type     = System<traits_type>;
    using forcefield_type = std::unique_ptr<ForceFieldBase<traits_type>>;
    using integrator_type = integratorT;

    static_assert(std::is_same<integratorT, VelocityVerletIntegrator<traitsT>>::value ||
                  std::is_same<integratorT, BAOABLangevinIntegrator<traitsT>>::value,
                  "B200Simulator runs VelocityVerlet or BAOABLangevin");

    // precision: MJG_PRECISION_FP64 (the reference's arithmetic) or
    // MJG_PRECISION_MIXED; seed: the Philox key of the Langevin noise
    // pair_inputs: by potential name, "ExcludedVolume", "DebyeHuckel", "LennardJones"
    B200Simulator(const std::size_t total_step, system_type&& sys, forcefield_type&& ff,
                  integrator_type&& integr, B200IgnoreRule ignore,
                  std::map<std::string, B200PairInput> pair_inputs, int precision = MJG_PRECISION_FP64,
                  std::uint64_t seed = 0, int device = 0)
        : total_step_(total_step), step_count_(0), system_(std::move(sys)), ff_(std::move(ff)),
          integrator_(std::move(integr)), ignore_(std::move(ignore)), pair_inputs_(std::move(pair_inputs)),
          precision_(precision), seed_(seed), device_(device)
    {}
    ~B200Simulator() override
    {
        if(ctx_) {mjg_context_destroy(ctx_);}
    }
    B200Simulator(const B200Simulator&) = delete;
    B200Simulator& operator=(const B200Simulator&) = delete;

    // MolecularDynamicsSimulator::initialize (core/MolecularDynamicsSimulator.hpp
    // :71-81): the system and the forcefield are initialised by the
    // reference's own code (topology, molecules, exclusion lists); then the
    // state and every interaction go to the GPU and the first forces are
    // computed there (mjg_commit).
    void initialize() override
    {
        system_.initialize(rng_);
        ff_->initialize(system_);
        check(mjg_context_create(device_, precision_, &ctx_), "mjg_context_create");
        upload_system();
        upload_forcefield();
        upload_integrator();
        check(mjg_commit(ctx_), "mjg_commit");
    }
    // one MD step (MolecularDynamicsSimulator::step, :83-102, without observers)
    bool step() override
    {
        check(mjg_step(ctx_, 1), "mjg_step");
        ++step_count_;
        return step_count_ < total_step_;
    }
    // every remaining step in one call
    void run() override
    {
        if(step_count_ < total_step_)
        {
            check(mjg_step(ctx_, static_cast<std::int64_t>(total_step_ - step_count_)), "mjg_step");
            step_count_ = total_step_;
        }
    }
    // the GPU state back into the reference System
    void finalize() override
    {
        const std::size_t n = system_.size();
        std::vector<double> p(3 * n), v(3 * n), f(3 * n);
        check(mjg_get_state(ctx_, id_, p.data(), v.data(), f.data()), "mjg_get_state");
        for(std::size_t i = 0; i < n; ++i)
        {
            system_.position(i) = coordinate_type(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
            system_.velocity(i) = coordinate_type(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
            system_.force(i)    = coordinate_type(f[3 * i], f[3 * i + 1], f[3 * i + 2]);
        }
    }
    // ForceField::calc_energy summed over the terms the GPU evaluates
    real_type calc_energy() const
    {
        double e[6] = {0, 0, 0, 0, 0, 0};
        check(mjg_energies(ctx_, id_, e), "mjg_energies");
        return e[0] + e[1] + e[2] + e[3] + e[4] + e[5];
    }

    system_type&       system()       noexcept {return system_;}
    system_type const& system() const noexcept {return system_;}
    forcefield_type&       forcefields()       noexcept {return ff_;}
    forcefield_type const& forcefields() const noexcept {return ff_;}

  private:
    static void check(int code, const char* what)
    {
        if(code != MJG_OK) {throw std::runtime_error(std::string("B200Simulator: ") + what + " failed (" +
                                                     std::to_string(code) + ")");}
    }

    // System<traits> (core/System.hpp:18-207): particles, boundary, attributes
    void upload_system()
    {
        const std::size_t n = system_.size();
        std::vector<double> p(3 * n), v(3 * n), m(n);
        for(std::size_t i = 0; i < n; ++i)
        {
            const auto& r = system_.position(i);
            const auto& u = system_.velocity(i);
            p[3 * i] = math::X(r); p[3 * i + 1] = math::Y(r); p[3 * i + 2] = math::Z(r);
            v[3 * i] = math::X(u); v[3 * i + 1] = math::Y(u); v[3 * i + 2] = math::Z(u);
            m[i] = system_.mass(i);
        }
        double lo[3] = {0, 0, 0}, up[3] = {0, 0, 0};
        const int boundary = box(system_.boundary(), lo, up);
        check(mjg_system_create(ctx_, static_cast<std::int64_t>(n), boundary, lo, up, p.data(), v.data(),
                                m.data(), &id_), "mjg_system_create");
        const real_type T = system_.has_attribute("temperature") ? system_.attribute("temperature") : real_type(300);
        const real_type I = system_.has_attribute("ionic_strength") ? system_.attribute("ionic_strength")
                                                                    : real_type(0.1);
        check(mjg_system_set_attributes(ctx_, id_, T, I), "mjg_system_set_attributes");
    }
    static int box(const UnlimitedBoundary<real_type, coordinate_type>&, double*, double*)
    {
        return MJG_UNLIMITED;
    }
    static int box(const CuboidalPeriodicBoundary<real_type, coordinate_type>& b, double* lo, double* up)
    {
        lo[0] = math::X(b.lower_bound()); lo[1] = math::Y(b.lower_bound()); lo[2] = math::Z(b.lower_bound());
        up[0] = math::X(b.upper_bound()); up[1] = math::Y(b.upper_bound()); up[2] = math::Z(b.upper_bound());
        return MJG_PERIODIC_CUBOID;
    }

    // every supported interaction of the ForceField (core/ForceField.hpp:165-170)
    void upload_forcefield()
    {
        const auto* ff = dynamic_cast<const ForceField<traits_type>*>(ff_.get());
        if(!ff) {throw std::runtime_error("B200Simulator: a ForceField<traits> is required");}
        if(!ff->external().empty()) {throw std::runtime_error("B200Simulator: external forcefields are not run");}

        std::vector<std::pair<std::size_t, std::size_t>> edges;   // candidate connections
        for(const auto& li : ff->local())
        {
            const auto* base = li.get();
            if(const auto* b = dynamic_cast<const BondLengthInteraction<traits_type, HarmonicPotential<real_type>>*>(base))
            {
                std::vector<std::int64_t> idx;
                std::vector<double> k, v0;
                for(const auto& t : b->potentials())
                {
                    idx.push_back(std::int64_t(t.first[0])); idx.push_back(std::int64_t(t.first[1]));
                    k.push_back(t.second.k()); v0.push_back(t.second.v0());
                    edges.emplace_back(t.first[0], t.first[1]);
                }
                check(mjg_bonds_set(ctx_, id_, "none", std::int64_t(k.size()), idx.data(), k.data(), v0.data()),
                      "mjg_bonds_set");
            }
            else if(const auto* a = dynamic_cast<const BondAngleInteraction<traits_type, HarmonicPotential<real_type>>*>(base))
            {
                std::vector<std::int64_t> idx;
                std::vector<double> k, v0;
                for(const auto& t : a->potentials())
                {
                    for(int x = 0; x < 3; ++x) {idx.push_back(std::int64_t(t.first[x]));}
                    k.push_back(t.second.k()); v0.push_back(t.second.v0());
                    edges.emplace_back(t.first[0], t.first[1]);
                    edges.emplace_back(t.first[1], t.first[2]);
                }
                check(mjg_angles_set(ctx_, id_, "none", std::int64_t(k.size()), idx.data(), k.data(), v0.data()),
                      "mjg_angles_set");
            }
            else if(const auto* d = dynamic_cast<const DihedralAngleInteraction<traits_type, CosinePotential<real_type>>*>(base))
            {
                std::vector<std::int64_t> idx;
                std::vector<double> k, v0;
                std::vector<std::int32_t> nn;
                for(const auto& t : d->potentials())
                {
                    for(int x = 0; x < 4; ++x) {idx.push_back(std::int64_t(t.first[x]));}
                    k.push_back(t.second.k()); nn.push_back(t.second.n()); v0.push_back(t.second.v0());
                    for(int x = 0; x < 3; ++x) {edges.emplace_back(t.first[x], t.first[x + 1]);}
                }
                check(mjg_dihedrals_set(ctx_, id_, "none", std::int64_t(k.size()), idx.data(), k.data(), nn.data(),
                                        v0.data()), "mjg_dihedrals_set");
            }
            else if(const auto* m = dynamic_cast<const DummyInteraction<traits_type>*>(base))
            {
                for(const auto& t : m->potentials()) {edges.emplace_back(t[0], t[1]);}
            }
            else
            {
                throw std::runtime_error("B200Simulator: unsupported local interaction " + base->name());
            }
        }
        upload_connections(ff->topology(), edges);

        for(const auto& gi : ff->global())
        {
            const auto* base = gi.get();
            if(const auto* e = dynamic_cast<const GlobalPairInteraction<traits_type, ExcludedVolumePotential<real_type>>*>(base))
            {
                const B200PairInput& in = pair_input("ExcludedVolume");
                const std::vector<std::int64_t> idx(in.participants.begin(), in.participants.end());
                check(mjg_exv_set(ctx_, id_, e->potential().epsilon(), e->potential().cutoff_ratio(),
                                  e->partition().margin(), std::int64_t(idx.size()), idx.data(), in.p0.data()),
                      "mjg_exv_set");
                set_ignore(MJG_TERM_EXV);
            }
            else if(const auto* h = dynamic_cast<const GlobalPairInteraction<traits_type, DebyeHuckelPotential<real_type>>*>(base))
            {
                const B200PairInput& in = pair_input("DebyeHuckel");
                const std::vector<std::int64_t> idx(in.participants.begin(), in.participants.end());
                check(mjg_dh_set(ctx_, id_, h->potential().cutoff_ratio(), h->partition().margin(),
                                 std::int64_t(idx.size()), idx.data(), in.p0.data()), "mjg_dh_set");
                set_ignore(MJG_TERM_DH);
            }
            else if(const auto* l = dynamic_cast<const GlobalPairInteraction<traits_type, LennardJonesPotential<real_type>>*>(base))
            {
                const B200PairInput& in = pair_input("LennardJones");
                const std::vector<std::int64_t> idx(in.participants.begin(), in.participants.end());
                check(mjg_lj_set(ctx_, id_, l->potential().cutoff_ratio(), l->partition().margin(),
                                 std::int64_t(idx.size()), idx.data(), in.p0.data(), in.p1.data()), "mjg_lj_set");
                set_ignore(MJG_TERM_LJ);
            }
            else
            {
                throw std::runtime_error("B200Simulator: unsupported global interaction " + base->name());
            }
        }
    }

    // the reference Topology's connections (core/Topology.hpp:45-125) between
    // every pair some local interaction joins, with their kinds
    void upload_connections(const Topology& topo, std::vector<std::pair<std::size_t, std::size_t>> edges)
    {
        for(auto& e : edges) {if(e.first > e.second) {std::swap(e.first, e.second);}}
        std::sort(edges.begin(), edges.end());
        edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
        std::map<std::string, std::vector<std::int64_t>> by_kind;
        for(const auto& e : edges)
        {
            for(const auto& kind : topo.list_connections_between(e.first, e.second))
            {
                by_kind[kind].push_back(std::int64_t(e.first));
                by_kind[kind].push_back(std::int64_t(e.second));
            }
        }
        for(const auto& kv : by_kind)
        {
            check(mjg_system_add_connections(ctx_, id_, kv.first.c_str(), std::int64_t(kv.second.size() / 2),
                                             kv.second.data()), "mjg_system_add_connections");
        }
    }

    const B200PairInput& pair_input(const std::string& name) const
    {
        const auto it = pair_inputs_.find(name);
        if(it == pair_inputs_.end()) {throw std::runtime_error("B200Simulator: no participants given for " + name);}
        return it->second;
    }

    void set_ignore(int term)
    {
        const int mol = ignore_.molecule == "Self"   || ignore_.molecule == "Intra" ? MJG_IGNORE_SELF   :
                        ignore_.molecule == "Others" || ignore_.molecule == "Inter" ? MJG_IGNORE_OTHERS :
                                                                                     MJG_IGNORE_NOTHING;
        std::vector<const char*> kinds;
        std::vector<std::int32_t> dist;
        for(const auto& kv : ignore_.within)
        {
            kinds.push_back(kv.first.c_str());
            dist.push_back(std::int32_t(kv.second));
        }
        check(mjg_ignore_set(ctx_, id_, term, mol, int(kinds.size()), kinds.data(), dist.data()), "mjg_ignore_set");
    }

    // integrator concept (core/BAOABLangevinIntegrator.hpp:34-69,
    // core/VelocityVerletIntegrator.hpp:15-60)
    void upload_integrator()
    {
        upload_integrator(integrator_);
    }
    void upload_integrator(const VelocityVerletIntegrator<traits_type>& vv)
    {
        check(mjg_integrator_set(ctx_, id_, MJG_VELOCITY_VERLET, vv.delta_t(), nullptr, seed_), "mjg_integrator_set");
    }
    void upload_integrator(const BAOABLangevinIntegrator<traits_type>& b)
    {
        std::vector<double> g(b.parameters().begin(), b.parameters().end());
        check(mjg_integrator_set(ctx_, id_, MJG_BAOAB, b.delta_t(), g.data(), seed_), "mjg_integrator_set");
    }

    std::size_t     total_step_;
    std::size_t     step_count_;
    system_type     system_;
    forcefield_type ff_;
    integrator_type integrator_;
    B200IgnoreRule  ignore_;
    std::map<std::string, B200PairInput> pair_inputs_;
    int             precision_;
    std::uint64_t   seed_;
    int             device_;
    RandomNumberGenerator<traits_type> rng_{0};   // System::initialize needs one; no noise drawn from it
    mjg_context*    ctx_ = nullptr;
    int             id_ = -1;
};

} // mjolnir
#endif // MJOLNIR_B200_SIMULATOR_HPP
