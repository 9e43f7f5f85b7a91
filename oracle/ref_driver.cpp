// TEST INFRASTRUCTURE ONLY -- not part of the product path.
//
// Drives the reference implementation itself: this translation unit includes
// the *unmodified* reference headers (found through -I<reference root>) and
// builds the reference's own objects from an orc_spec, so that the tests and
// the CPU-baseline leg of bench.py can ask the reference for
//   - per-term forces and energies   (GlobalPair*Interaction / Bond*Interaction
//                                     ::calc_force_and_energy, calc_energy),
//   - its half neighbour lists       (SpatialPartition::neighbors(), the CSR of
//                                     core/NeighborList.hpp:151-266),
//   - trajectories                   (BAOABLangevinIntegrator::step,
//                                     VelocityVerletIntegrator::step,
//                                     UnderdampedLangevinIntegrator::step,
//                                     GJFNVTLangevinIntegrator::step,
//                                     gBAOABLangevinIntegrator::step),
//   - timings of its sequential and OpenMP paths.
// The objects are put together the way the input readers do it
// (input/read_global_interaction.hpp:25-98, input/read_local_interaction.hpp,
//  input/read_integrator.hpp:120-187, input/read_system.hpp:93-290) because
// toml11 is not available to run those readers directly.
// Built by oracle/Makefile into oracle/_ref/libmjolnir_ref.so.

#include <mjolnir/util/logger.hpp>
#include <mjolnir/core/SimulatorTraits.hpp>
#include <mjolnir/core/BoundaryCondition.hpp>
#include <mjolnir/core/System.hpp>
#include <mjolnir/core/ForceField.hpp>
#include <mjolnir/core/Unit.hpp>
#include <mjolnir/core/MsgPackSaver.hpp>
#include <mjolnir/core/MsgPackLoader.hpp>
#include <mjolnir/core/XYZObserver.hpp>
#include <mjolnir/core/DCDObserver.hpp>
#include <mjolnir/core/TRRObserver.hpp>
#include <mjolnir/core/EnergyObserver.hpp>
#include <mjolnir/core/BAOABLangevinIntegrator.hpp>
#include <mjolnir/core/VelocityVerletIntegrator.hpp>
#include <mjolnir/core/UnderdampedLangevinIntegrator.hpp>
#include <mjolnir/core/GJFNVTLangevinIntegrator.hpp>
#include <mjolnir/core/gBAOABLangevinIntegrator.hpp>
#include <mjolnir/core/PeriodicGridCellList.hpp>
#include <mjolnir/core/UnlimitedGridCellList.hpp>
#include <mjolnir/forcefield/global/GlobalPairInteraction.hpp>
#include <mjolnir/forcefield/global/GlobalPairExcludedVolumeInteraction.hpp>
#include <mjolnir/forcefield/global/GlobalPairLennardJonesInteraction.hpp>
#include <mjolnir/forcefield/global/ExcludedVolumePotential.hpp>
#include <mjolnir/forcefield/global/DebyeHuckelPotential.hpp>
#include <mjolnir/forcefield/global/LennardJonesPotential.hpp>
#include <mjolnir/forcefield/global/WCAPotential.hpp>
#include <mjolnir/forcefield/global/InversePowerPotential.hpp>
#include <mjolnir/forcefield/global/HardCoreExcludedVolumePotential.hpp>
#include <mjolnir/forcefield/global/LennardJonesAttractivePotential.hpp>
#include <mjolnir/forcefield/global/UniformLennardJonesPotential.hpp>
#include <mjolnir/forcefield/local/BondLengthInteraction.hpp>
#include <mjolnir/forcefield/local/BondAngleInteraction.hpp>
#include <mjolnir/forcefield/local/DihedralAngleInteraction.hpp>
#include <mjolnir/forcefield/local/DummyInteraction.hpp>
#include <mjolnir/forcefield/local/HarmonicPotential.hpp>
#include <mjolnir/forcefield/local/CosinePotential.hpp>
#ifdef MJOLNIR_WITH_OPENMP
#include <mjolnir/omp/omp.hpp>
#endif

#include "spec.h"
#include <chrono>
#include <cstring>
#include <memory>
#include <string>

namespace
{
using namespace mjolnir;

thread_local std::string g_error;

// Units exactly as read_units sets them for energy "kcal/mol", length
// "angstrom" (input/read_units.hpp:32-91).
void set_units_once()
{
    static bool done = false;
    if(done) {return;}
    done = true;
    LoggerManager::set_default_logger("/dev/null");

    using phys_type = physics::constants<double>;
    using unit_type = unit::constants<double>;
    // the constants are process-wide (template statics are shared by every
    // library that includes the reference headers): convert them only once
    if(phys_type::energy_unit() == "kcal/mol") {return;}
    phys_type::set_kB(phys_type::kB() * (unit_type::J_to_cal() / 1000.0) *
                      unit_type::avogadro_constant());
    phys_type::set_eps0(phys_type::eps0() * (1000.0 / unit_type::J_to_cal()) /
                        unit_type::avogadro_constant());
    phys_type::set_eps0(phys_type::eps0() / unit_type::m_to_angstrom());
    phys_type::set_m_to_length(unit_type::m_to_angstrom());
    phys_type::set_length_to_m(unit_type::angstrom_to_m());
    phys_type::set_L_to_volume(1e-3 * std::pow(unit_type::m_to_angstrom(), 3));
    phys_type::set_volume_to_L(1e+3 * std::pow(unit_type::angstrom_to_m(), 3));
    phys_type::set_energy_unit("kcal/mol");
    phys_type::set_length_unit("angstrom");
}

struct RefSimBase
{
    virtual ~RefSimBase() = default;
    virtual int  term_force(int term, double* force, double* energy) = 0;
    virtual int  term_energy(int term, double* energy) = 0;
    virtual long long neighbors(int term, long long* pairs, long long cap) = 0;
    virtual void initialize() = 0;
    virtual void run(long long nsteps) = 0;
    virtual void get_state(double* pos, double* vel, double* force) = 0;
    virtual void total_force(double* force) = 0;
    virtual double total_energy() = 0;
    virtual void save_msgpack(const std::string& prefix) = 0;
    virtual void observe(const std::string& prefix, int formats, long long total_step,
                         long long save_step, double dt) = 0;
};

template<typename coordT>
coordT make_xyz(const double* p) {return coordT(p[0], p[1], p[2]);}

template<typename traitsT, bool Sequential>
struct RefSim final : public RefSimBase
{
    using real_type       = double;
    using coordinate_type = typename traitsT::coordinate_type;
    using boundary_type   = typename traitsT::boundary_type;
    using system_type     = System<traitsT>;
    using ff_base_type    = ForceFieldBase<traitsT>;
    using rng_type        = RandomNumberGenerator<traitsT>;
    using local_base      = LocalInteractionBase<traitsT>;
    using global_base     = GlobalInteractionBase<traitsT>;
    using remover_type    = SystemMotionRemover<traitsT>;

    using exv_pot = ExcludedVolumePotential<double>;
    using dh_pot  = DebyeHuckelPotential<double>;
    using lj_pot  = LennardJonesPotential<double>;
    using wca_pot = WCAPotential<double>;
    using lja_pot = LennardJonesAttractivePotential<double>;
    using ulj_pot = UniformLennardJonesPotential<double>;
    using ipw_pot = InversePowerPotential<double>;
    using hcx_pot = HardCoreExcludedVolumePotential<double>;
    int lj_kind = ORC_LJ;
    int exv_kind = ORC_EXV;

    std::unique_ptr<system_type>  sys;
    std::unique_ptr<ff_base_type> ff;
    rng_type rng;
    std::unique_ptr<BAOABLangevinIntegrator<traitsT>> baoab;
    std::unique_ptr<VelocityVerletIntegrator<traitsT>> vv;
    std::unique_ptr<UnderdampedLangevinIntegrator<traitsT>> ul;
    std::unique_ptr<GJFNVTLangevinIntegrator<traitsT>> gjf;
    std::unique_ptr<gBAOABLangevinIntegrator<traitsT>> gbaoab;
    local_base*  locals [3] = {nullptr, nullptr, nullptr};
    global_base* globals[3] = {nullptr, nullptr, nullptr};
    double time = 0.0;
    std::vector<std::size_t> leading[3];

    static boundary_type make_boundary(const orc_spec& s, std::true_type)
    {
        return boundary_type(make_xyz<coordinate_type>(s.lower),
                             make_xyz<coordinate_type>(s.upper));
    }
    static boundary_type make_boundary(const orc_spec&, std::false_type)
    {
        return boundary_type();
    }

    template<typename potT>
    static SpatialPartition<traitsT, potT> make_partition(double margin, std::true_type)
    {
        return SpatialPartition<traitsT, potT>(
            make_unique<PeriodicGridCellList<traitsT, potT>>(margin));
    }
    template<typename potT>
    static SpatialPartition<traitsT, potT> make_partition(double margin, std::false_type)
    {
        return SpatialPartition<traitsT, potT>(
            make_unique<UnlimitedGridCellList<traitsT, potT>>(margin));
    }

    explicit RefSim(const orc_spec& s)
        : rng(static_cast<std::uint32_t>(s.seed))
    {
        using is_periodic = is_cuboidal_periodic_boundary<boundary_type>;
        const std::size_t N = static_cast<std::size_t>(s.n);

        sys = make_unique<system_type>(N, make_boundary(s, is_periodic{}));
        for(std::size_t i=0; i<N; ++i)
        {
            sys->mass(i)     = s.mass[i];
            sys->rmass(i)    = 1.0 / s.mass[i];      // read_system.hpp:279
            sys->position(i) = make_xyz<coordinate_type>(s.pos + 3*i);
            sys->velocity(i) = make_xyz<coordinate_type>(s.vel + 3*i);
            sys->force(i)    = coordinate_type(0, 0, 0);
            sys->name(i)     = "X";
            sys->group(i)    = "NONE";               // read_system.hpp:278
        }
        sys->velocity_initialized() = true;
        sys->attribute("temperature")    = s.temperature;
        sys->attribute("ionic_strength") = s.ionic_strength;
        sys->initialize(rng);   // wraps positions into the box

        // ------------------------------------------------------------- local
        LocalForceField<traitsT> local;
        if(s.nbond > 0)
        {
            using pot = HarmonicPotential<double>;
            using inter = BondLengthInteraction<traitsT, pot>;
            typename inter::container_type c;
            for(long long b=0; b<s.nbond; ++b)
            {
                c.emplace_back(typename inter::indices_type{{
                    std::size_t(s.bond_idx[2*b]), std::size_t(s.bond_idx[2*b+1])}},
                    pot(s.bond_k[b], s.bond_v0[b]));
            }
            auto p = make_unique<inter>("bond", std::move(c));
            locals[ORC_TERM_BOND] = p.get();
            local.emplace(std::move(p));
        }
        if(s.nangle > 0)
        {
            using pot = HarmonicPotential<double>;
            using inter = BondAngleInteraction<traitsT, pot>;
            typename inter::container_type c;
            for(long long b=0; b<s.nangle; ++b)
            {
                c.emplace_back(typename inter::indices_type{{
                    std::size_t(s.angle_idx[3*b]), std::size_t(s.angle_idx[3*b+1]),
                    std::size_t(s.angle_idx[3*b+2])}},
                    pot(s.angle_k[b], s.angle_v0[b]));
            }
            auto p = make_unique<inter>("none", std::move(c));
            locals[ORC_TERM_ANGLE] = p.get();
            local.emplace(std::move(p));
        }
        if(s.ndihd > 0)
        {
            using pot = CosinePotential<double>;
            using inter = DihedralAngleInteraction<traitsT, pot>;
            typename inter::container_type c;
            for(long long b=0; b<s.ndihd; ++b)
            {
                c.emplace_back(typename inter::indices_type{{
                    std::size_t(s.dihd_idx[4*b]),   std::size_t(s.dihd_idx[4*b+1]),
                    std::size_t(s.dihd_idx[4*b+2]), std::size_t(s.dihd_idx[4*b+3])}},
                    pot(s.dihd_k[b], s.dihd_n[b], s.dihd_v0[b]));
            }
            auto p = make_unique<inter>("none", std::move(c));
            locals[ORC_TERM_DIHEDRAL] = p.get();
            local.emplace(std::move(p));
        }
        if(s.single_molecule && N > 1)
        {
            typename DummyInteraction<traitsT>::container_type c;
            for(std::size_t i=0; i+1<N; ++i) {c.push_back({{i, i+1}});}
            local.emplace(make_unique<DummyInteraction<traitsT>>("bond", c));
        }

        // ------------------------------------------------------------ global
        const long long     np[3] = {s.exv_on ? s.exv_n : 0, s.dh_on ? s.dh_n : 0, s.lj_on ? s.lj_n : 0};
        const int64_t* const ip[3] = {s.exv_idx, s.dh_idx, s.lj_idx};
        for(int g=0; g<3; ++g)
        {
            for(long long k=0; k+1<np[g]; ++k) {leading[g].push_back(std::size_t(ip[g][k]));}
        }
        std::map<std::string, std::size_t> within;
        if(s.ignore_bond_within > 0) {within["bond"] = std::size_t(s.ignore_bond_within);}
        const char* mol_rule = s.ignore_molecule == ORC_IGNORE_SELF   ? "Self"   :
                               s.ignore_molecule == ORC_IGNORE_OTHERS ? "Others" :
                                                                        "Nothing";
        GlobalForceField<traitsT> global;
        exv_kind = s.exv_kind;
        if(s.exv_on && s.exv_kind == ORC_INVERSE_POWER)
        {
            using plist = InversePowerParameterList<traitsT>;
            std::vector<std::pair<std::size_t, typename plist::parameter_type>> ps;
            for(long long k=0; k<s.exv_n; ++k)
            {
                ps.emplace_back(std::size_t(s.exv_idx[k]), typename plist::parameter_type{s.exv_radius[k]});
            }
            auto p = make_unique<GlobalPairInteraction<traitsT, ipw_pot>>(
                ipw_pot(s.exv_cutoff, s.exv_power, s.exv_eps),
                ParameterList<traitsT, ipw_pot>(make_unique<plist>(ps, within, IgnoreMolecule<std::size_t>(mol_rule),
                    IgnoreGroup<std::string>(std::map<std::string, std::vector<std::string>>{}))),
                make_partition<ipw_pot>(s.exv_margin, is_periodic{}));
            globals[0] = p.get();
            global.emplace(std::move(p));
        }
        else if(s.exv_on && s.exv_kind == ORC_HARD_CORE_EXV)
        {
            using plist = HardCoreExcludedVolumeParameterList<traitsT>;
            std::vector<std::pair<std::size_t, typename plist::parameter_type>> ps;
            for(long long k=0; k<s.exv_n; ++k)
            {
                ps.emplace_back(std::size_t(s.exv_idx[k]),
                                typename plist::parameter_type{s.exv_radius[k], s.exv_core[k]});
            }
            auto p = make_unique<GlobalPairInteraction<traitsT, hcx_pot>>(
                hcx_pot(s.exv_cutoff, s.exv_eps),
                ParameterList<traitsT, hcx_pot>(make_unique<plist>(ps, within, IgnoreMolecule<std::size_t>(mol_rule),
                    IgnoreGroup<std::string>(std::map<std::string, std::vector<std::string>>{}))),
                make_partition<hcx_pot>(s.exv_margin, is_periodic{}));
            globals[0] = p.get();
            global.emplace(std::move(p));
        }
        else if(s.exv_on)
        {
            using plist = ExcludedVolumeParameterList<traitsT>;
            std::vector<std::pair<std::size_t, typename plist::parameter_type>> ps;
            for(long long k=0; k<s.exv_n; ++k)
            {
                ps.emplace_back(std::size_t(s.exv_idx[k]),
                                typename plist::parameter_type{s.exv_radius[k]});
            }
            auto p = make_unique<GlobalPairInteraction<traitsT, exv_pot>>(
                exv_pot(s.exv_cutoff, s.exv_eps),
                ParameterList<traitsT, exv_pot>(make_unique<plist>(ps, within,
                    IgnoreMolecule<std::size_t>(mol_rule),
                    IgnoreGroup<std::string>(std::map<std::string, std::vector<std::string>>{}))),
                make_partition<exv_pot>(s.exv_margin, is_periodic{}));
            globals[0] = p.get();
            global.emplace(std::move(p));
        }
        if(s.dh_on)
        {
            using plist = DebyeHuckelParameterList<traitsT>;
            std::vector<std::pair<std::size_t, typename plist::parameter_type>> ps;
            for(long long k=0; k<s.dh_n; ++k)
            {
                ps.emplace_back(std::size_t(s.dh_idx[k]),
                                typename plist::parameter_type{s.dh_charge[k]});
            }
            auto p = make_unique<GlobalPairInteraction<traitsT, dh_pot>>(
                dh_pot(s.dh_cutoff),
                ParameterList<traitsT, dh_pot>(make_unique<plist>(ps, within,
                    IgnoreMolecule<std::size_t>(mol_rule),
                    IgnoreGroup<std::string>(std::map<std::string, std::vector<std::string>>{}))),
                make_partition<dh_pot>(s.dh_margin, is_periodic{}));
            globals[1] = p.get();
            global.emplace(std::move(p));
        }
        lj_kind = s.lj_kind;
        if(s.lj_on && s.lj_kind != ORC_LJ)
        {
            add_lj_family(s, global, within, mol_rule, is_periodic{});
        }
        else if(s.lj_on)
        {
            using plist = LorentzBerthelotRule<traitsT, lj_pot>;
            std::vector<std::pair<std::size_t, typename plist::parameter_type>> ps;
            for(long long k=0; k<s.lj_n; ++k)
            {
                ps.emplace_back(std::size_t(s.lj_idx[k]),
                    typename plist::parameter_type{s.lj_sigma[k], s.lj_eps[k]});
            }
            auto p = make_unique<GlobalPairInteraction<traitsT, lj_pot>>(
                lj_pot(s.lj_cutoff),
                ParameterList<traitsT, lj_pot>(make_unique<plist>(ps, within,
                    IgnoreMolecule<std::size_t>(mol_rule),
                    IgnoreGroup<std::string>(std::map<std::string, std::vector<std::string>>{}))),
                make_partition<lj_pot>(s.lj_margin, is_periodic{}));
            globals[2] = p.get();
            global.emplace(std::move(p));
        }

        ff = make_unique<ForceField<traitsT>>(std::move(local), std::move(global),
                ExternalForceField<traitsT>{}, ConstraintForceField<traitsT>{});
        ff->initialize(*sys);   // topology, exclusion lists, first list build

        std::vector<double> gam(s.gamma, s.gamma + N);
        if(s.integrator == ORC_VV)
        {
            make_vv(s.dt, std::integral_constant<bool, Sequential>{});
        }
        else if(s.integrator == ORC_UNDERDAMPED)
        {
            ul = make_unique<UnderdampedLangevinIntegrator<traitsT>>(s.dt,
                        std::move(gam), remover_type(false, false, false));
        }
        else if(s.integrator == ORC_GJF)
        {
            gjf = make_unique<GJFNVTLangevinIntegrator<traitsT>>(s.dt,
                        std::move(gam), remover_type(false, false, false));
        }
        else if(s.integrator == ORC_GBAOAB)
        {
            gbaoab = make_unique<gBAOABLangevinIntegrator<traitsT>>(s.dt,
                        std::move(gam), remover_type(false, false, false));
        }
        else
        {
            baoab = make_unique<BAOABLangevinIntegrator<traitsT>>(s.dt,
                        std::move(gam), remover_type(false, false, false));
        }
    }

    void make_vv(double dt, std::true_type)
    {
        vv = make_unique<VelocityVerletIntegrator<traitsT>>(dt,
                remover_type(false, false, false));
    }
    void make_vv(double, std::false_type)
    {
        throw std::runtime_error("the reference has no OpenMP velocity Verlet");
    }

    void zero_force()
    {
        for(std::size_t i=0; i<sys->size(); ++i)
        {
            sys->force(i) = coordinate_type(0, 0, 0);
        }
    }
    void copy_force(double* out)
    {
        for(std::size_t i=0; i<sys->size(); ++i)
        {
            const auto& f = sys->force(i);
            out[3*i+0] = math::X(f); out[3*i+1] = math::Y(f); out[3*i+2] = math::Z(f);
        }
    }

    int term_force(int term, double* force, double* energy) override
    {
        zero_force();
        double e = 0.0;
        sys->preprocess_forces();
        if(term <= ORC_TERM_DIHEDRAL)
        {
            if(!locals[term]) {return -1;}
            e = locals[term]->calc_force_and_energy(*sys);
        }
        else
        {
            if(!globals[term - ORC_TERM_EXV]) {return -1;}
            e = globals[term - ORC_TERM_EXV]->calc_force_and_energy(*sys);
        }
        sys->postprocess_forces();
        copy_force(force);
        *energy = e;
        return 0;
    }
    int term_energy(int term, double* energy) override
    {
        if(term <= ORC_TERM_DIHEDRAL)
        {
            if(!locals[term]) {return -1;}
            *energy = locals[term]->calc_energy(*sys);
        }
        else
        {
            if(!globals[term - ORC_TERM_EXV]) {return -1;}
            *energy = globals[term - ORC_TERM_EXV]->calc_energy(*sys);
        }
        return 0;
    }

    // partners(i) is valid only for leading participants (every participant
    // but the last one, ParameterList.hpp leading_participants()).
    template<typename potT>
    long long dump(global_base* g, const std::vector<std::size_t>& leading,
                   long long* pairs, long long cap, std::true_type)
    {
        auto* gp = dynamic_cast<GlobalPairInteraction<traitsT, potT>*>(g);
        if(!gp) {return -1;}
        const auto& part = gp->partition();
        long long k = 0;
        for(const std::size_t i : leading)
        {
            for(const auto& nb : part.partners(i))
            {
                if(k < cap) {pairs[2*k] = (long long)i; pairs[2*k+1] = (long long)nb.index;}
                ++k;
            }
        }
        return k;
    }
    template<typename potT>
    long long dump(global_base*, const std::vector<std::size_t>&, long long*,
                   long long, std::false_type) {return -1;}

    // WCA / LennardJonesAttractive (Lorentz-Berthelot parameters) and
    // UniformLennardJones (one sigma and epsilon) through the generic
    // GlobalPairInteraction, as input/read_global_potential.hpp builds them
    template<typename potT, typename withinT, typename molT, typename periodicT>
    void add_lb(const orc_spec& s, potT pot, GlobalForceField<traitsT>& global, const withinT& within,
                const molT& mol_rule, periodicT per)
    {
        using plist = LorentzBerthelotRule<traitsT, potT>;
        std::vector<std::pair<std::size_t, typename plist::parameter_type>> ps;
        for(long long k=0; k<s.lj_n; ++k)
        {
            ps.emplace_back(std::size_t(s.lj_idx[k]), typename plist::parameter_type{s.lj_sigma[k], s.lj_eps[k]});
        }
        auto p = make_unique<GlobalPairInteraction<traitsT, potT>>(std::move(pot),
            ParameterList<traitsT, potT>(make_unique<plist>(ps, within, IgnoreMolecule<std::size_t>(mol_rule),
                IgnoreGroup<std::string>(std::map<std::string, std::vector<std::string>>{}))),
            make_partition<potT>(s.lj_margin, per));
        globals[2] = p.get();
        global.emplace(std::move(p));
    }
    template<typename withinT, typename molT, typename periodicT>
    void add_lj_family(const orc_spec& s, GlobalForceField<traitsT>& global, const withinT& within,
                       const molT& mol_rule, periodicT per)
    {
        if(s.lj_kind == ORC_WCA)                {add_lb(s, wca_pot(), global, within, mol_rule, per); return;}
        if(s.lj_kind == ORC_LJ_ATTRACTIVE)      {add_lb(s, lja_pot(s.lj_cutoff), global, within, mol_rule, per); return;}
        using plist = EmptyCombinationRule<traitsT, ulj_pot>;
        std::vector<std::size_t> parts;
        for(long long k=0; k<s.lj_n; ++k) {parts.push_back(std::size_t(s.lj_idx[k]));}
        auto p = make_unique<GlobalPairInteraction<traitsT, ulj_pot>>(
            ulj_pot(s.lj_cutoff, s.lj_n > 0 ? s.lj_sigma[0] : 1.0, s.lj_n > 0 ? s.lj_eps[0] : 1.0),
            ParameterList<traitsT, ulj_pot>(make_unique<plist>(parts, within, IgnoreMolecule<std::size_t>(mol_rule),
                IgnoreGroup<std::string>(std::map<std::string, std::vector<std::string>>{}))),
            make_partition<ulj_pot>(s.lj_margin, per));
        globals[2] = p.get();
        global.emplace(std::move(p));
    }

    long long neighbors(int term, long long* pairs, long long cap) override
    {
        const int g = term - ORC_TERM_EXV;
        if(g < 0 || g > 2 || !globals[g]) {return -1;}
        std::integral_constant<bool, Sequential> seq;
        if(g == 0)
        {
            if(exv_kind == ORC_INVERSE_POWER) {return dump<ipw_pot>(globals[0], leading[0], pairs, cap, seq);}
            if(exv_kind == ORC_HARD_CORE_EXV) {return dump<hcx_pot>(globals[0], leading[0], pairs, cap, seq);}
            return dump<exv_pot>(globals[0], leading[0], pairs, cap, seq);
        }
        if(g == 1) {return dump<dh_pot >(globals[1], leading[1], pairs, cap, seq);}
        if(lj_kind == ORC_WCA)           {return dump<wca_pot>(globals[2], leading[2], pairs, cap, seq);}
        if(lj_kind == ORC_LJ_ATTRACTIVE) {return dump<lja_pot>(globals[2], leading[2], pairs, cap, seq);}
        if(lj_kind == ORC_LJ_UNIFORM)    {return dump<ulj_pot>(globals[2], leading[2], pairs, cap, seq);}
        return dump<lj_pot>(globals[2], leading[2], pairs, cap, seq);
    }

    void initialize() override
    {
        if(baoab)   {baoab->initialize(*sys, ff, rng);}
        else if(ul) {ul->initialize(*sys, ff, rng);}
        else if(gjf){gjf->initialize(*sys, ff, rng);}
        else if(gbaoab) {gbaoab->initialize(*sys, ff, rng);}
        else        {vv->initialize(*sys, ff, rng);}
    }
    void run(long long nsteps) override
    {
        for(long long s=0; s<nsteps; ++s)
        {
            time = baoab ? baoab->step(time, *sys, ff, rng)
                 : ul    ? ul->step(time, *sys, ff, rng)
                 : gjf   ? gjf->step(time, *sys, ff, rng)
                 : gbaoab ? gbaoab->step(time, *sys, ff, rng)
                         : vv->step(time, *sys, ff, rng);
        }
    }
    // MolecularDynamicsSimulator::initialize / step / finalize
    // (core/MolecularDynamicsSimulator.hpp:72-125) with the observers that
    // read_observer builds (input/read_observer.hpp:17-96): formats bit 0 xyz,
    // bit 1 dcd, bit 2 trr; the energy file always.  The integrator must have
    // been initialised.
    void observe(const std::string& prefix, int formats, long long total_step,
                 long long save_step, double dt) override
    {
        std::vector<std::unique_ptr<ObserverBase<traitsT>>> obs;
        if(formats & 1) {obs.push_back(make_unique<XYZObserver<traitsT>>(prefix));}
        if(formats & 2) {obs.push_back(make_unique<DCDObserver<traitsT>>(prefix));}
        if(formats & 4) {obs.push_back(make_unique<TRRObserver<traitsT>>(prefix));}
        obs.push_back(make_unique<EnergyObserver<traitsT>>(prefix));
        for(auto& o : obs) {o->initialize(total_step, save_step, dt, *sys, ff);}
        for(long long st = 0; st < total_step; ++st)
        {
            if(st % save_step == 0) {for(auto& o : obs) {o->output(st, dt, *sys, ff);}}
            run(1);
        }
        for(auto& o : obs) {o->output(total_step, dt, *sys, ff);}
        for(auto& o : obs) {o->finalize(total_step, dt, *sys, ff);}
    }
    // MsgPackSaver::save(System) writes prefix + "_system.msg"
    void save_msgpack(const std::string& prefix) override
    {
        MsgPackSaver<traitsT> saver(prefix);
        saver.save(*sys);
    }

    void get_state(double* pos, double* vel, double* force) override
    {
        for(std::size_t i=0; i<sys->size(); ++i)
        {
            const auto& p = sys->position(i);
            const auto& v = sys->velocity(i);
            if(pos) {pos[3*i] = math::X(p); pos[3*i+1] = math::Y(p); pos[3*i+2] = math::Z(p);}
            if(vel) {vel[3*i] = math::X(v); vel[3*i+1] = math::Y(v); vel[3*i+2] = math::Z(v);}
        }
        if(force) {copy_force(force);}
    }
    void total_force(double* force) override
    {
        zero_force();
        ff->calc_force(*sys);
        copy_force(force);
    }
    double total_energy() override
    {
        return ff->calc_energy(*sys);
    }
};

template<template<typename, template<typename, typename> class> class traitsT, bool Seq>
RefSimBase* make_sim(const orc_spec& s)
{
    if(s.boundary == ORC_PERIODIC)
    {
        return new RefSim<traitsT<double, CuboidalPeriodicBoundary>, Seq>(s);
    }
    return new RefSim<traitsT<double, UnlimitedBoundary>, Seq>(s);
}

template<typename sysT>
long long copy_system(const sysT& sys, long long cap, double* pos, double* vel, double* force,
                      double* mass, double* temperature, double* ionic_strength)
{
    const long long n = (long long)sys.size();
    for(long long i = 0; i < n && i < cap; ++i)
    {
        for(int x = 0; x < 3; ++x)
        {
            pos[3 * i + x]   = sys.position(i)[x];
            vel[3 * i + x]   = sys.velocity(i)[x];
            force[3 * i + x] = sys.force(i)[x];
        }
        mass[i] = sys.mass(i);
    }
    const auto& at = sys.attributes();
    *temperature    = at.count("temperature")    ? at.at("temperature")    : 0.0;
    *ionic_strength = at.count("ionic_strength") ? at.at("ionic_strength") : 0.0;
    return n;
}

} // anonymous

extern "C" {

const char* ref_last_error(void) {return g_error.c_str();}

// parallel: 0 = SimulatorTraits (sequential), 1 = OpenMPSimulatorTraits.
void* ref_create(const orc_spec* spec, int parallel)
{
    try
    {
        set_units_once();
        if(parallel)
        {
#ifdef MJOLNIR_WITH_OPENMP
            return make_sim<OpenMPSimulatorTraits, false>(*spec);
#else
            g_error = "built without OpenMP";
            return nullptr;
#endif
        }
        return make_sim<SimulatorTraits, true>(*spec);
    }
    catch(const std::exception& e)
    {
        g_error = e.what();
        return nullptr;
    }
}
void ref_destroy(void* h) {delete static_cast<RefSimBase*>(h);}

int ref_term_force(void* h, int term, double* force, double* energy)
{
    return static_cast<RefSimBase*>(h)->term_force(term, force, energy);
}
int ref_term_energy(void* h, int term, double* energy)
{
    return static_cast<RefSimBase*>(h)->term_energy(term, energy);
}
long long ref_neighbors(void* h, int term, long long* pairs, long long cap)
{
    return static_cast<RefSimBase*>(h)->neighbors(term, pairs, cap);
}
void ref_initialize(void* h) {static_cast<RefSimBase*>(h)->initialize();}

// Runs nsteps integrator steps and returns the wall time of the loop in seconds.
double ref_run(void* h, long long nsteps)
{
    const auto t0 = std::chrono::steady_clock::now();
    static_cast<RefSimBase*>(h)->run(nsteps);
    const auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}
void ref_get_state(void* h, double* pos, double* vel, double* force)
{
    static_cast<RefSimBase*>(h)->get_state(pos, vel, force);
}
void ref_total_force(void* h, double* force) {static_cast<RefSimBase*>(h)->total_force(force);}
double ref_total_energy(void* h) {return static_cast<RefSimBase*>(h)->total_energy();}

// The reference's checkpoint writer on the current system state.
int ref_observe(void* h, const char* prefix, int formats, long long total_step,
                long long save_step, double dt)
{
    try
    {
        static_cast<RefSimBase*>(h)->observe(prefix, formats, total_step, save_step, dt);
        return 0;
    }
    catch(const std::exception& e)
    {
        g_error = e.what();
        return -1;
    }
}

int ref_save_msgpack(void* h, const char* prefix)
{
    try
    {
        static_cast<RefSimBase*>(h)->save_msgpack(prefix);
        return 0;
    }
    catch(const std::exception& e)
    {
        g_error = e.what();
        return -1;
    }
}

// The reference's checkpoint reader (MsgPackLoader::load_system): copies out
// what it read.  periodic selects the boundary type the file must hold.
// Returns the number of particles, or -1 (ref_last_error) on failure; copies
// at most cap particles.
long long ref_load_msgpack(const char* file, int periodic, long long cap, double* pos,
                           double* vel, double* force, double* mass, double* lower,
                           double* upper, double* temperature, double* ionic_strength)
{
    try
    {
        if(periodic)
        {
            MsgPackLoader<SimulatorTraits<double, CuboidalPeriodicBoundary>> loader;
            const auto sys = loader.load_system(file);
            for(int x = 0; x < 3; ++x)
            {
                lower[x] = sys.boundary().lower_bound()[x];
                upper[x] = sys.boundary().upper_bound()[x];
            }
            return copy_system(sys, cap, pos, vel, force, mass, temperature, ionic_strength);
        }
        MsgPackLoader<SimulatorTraits<double, UnlimitedBoundary>> loader;
        const auto sys = loader.load_system(file);
        return copy_system(sys, cap, pos, vel, force, mass, temperature, ionic_strength);
    }
    catch(const std::exception& e)
    {
        g_error = e.what();
        return -1;
    }
}

int ref_max_threads(void)
{
#ifdef MJOLNIR_WITH_OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

} // extern "C"
