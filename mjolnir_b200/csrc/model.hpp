// Host-side model set-up shared by the context: unit constants, the
// Debye-Hueckel parameters, the topology (molecules) and the per-particle
// exclusion lists.  These run once per commit, on the CPU, in the reference's
// operation order so that the GPU sees the same constants.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <string>
#include <utility>
#include <vector>

namespace mjg {

// core/Unit.hpp:23-26,150-156 followed by input/read_units.hpp:32-91
// (energy "kcal/mol", length "angstrom").
struct Units {
    double kB, NA, eps0, L_to_volume;
    Units()
    {
        const double boltzmann   = 1.38064852e-23;
        const double avogadro    = 6.022140857e23;
        const double e_charge    = 1.6021766208e-19;
        const double vacuum_perm = 8.854187817e-12;
        const double J_to_cal    = 1.0 / 4.184;
        const double m_to_ang    = 1e+10;
        kB   = boltzmann;
        eps0 = (vacuum_perm / e_charge) / e_charge;
        kB   = kB * (J_to_cal / 1000.0) * avogadro;
        eps0 = eps0 * (1000.0 / J_to_cal) / avogadro;
        eps0 = eps0 / m_to_ang;
        NA   = avogadro;
        L_to_volume = 1e-3 * std::pow(m_to_ang, 3);
    }
};

// DebyeHuckelPotential::calc_parameters and calc_dielectric_water
// (forcefield/global/DebyeHuckelPotential.hpp:126-174).
struct DHParams {
    double debye, inv_debye, abs_cutoff, coef_at_cutoff, inv4pi;
};
inline DHParams dh_params(double T, double c, double cutoff_ratio)
{
    const Units u;
    const double pi   = 3.14159265358979323846264338;
    const double epsk = (249.4 - 0.788 * T + 7.2e-4 * T * T) *
                        (1. - 2.551e-1 * c + 5.151e-2 * c * c - 6.889e-3 * c * c * c);
    DHParams p;
    p.inv4pi     = 1.0 / (4 * pi * u.eps0 * epsk);
    const double I = c / u.L_to_volume;
    p.debye      = std::sqrt((u.eps0 * epsk * u.kB * T) / (2 * u.NA * I));
    p.inv_debye  = 1. / p.debye;
    p.abs_cutoff = cutoff_ratio * p.debye;
    p.coef_at_cutoff = std::exp(-cutoff_ratio) / (p.debye * cutoff_ratio);
    return p;
}

// Connection graph of one system (core/Topology.hpp): adjacency lists in
// insertion order, duplicate edges of the same kind dropped.
class TopologyGraph {
  public:
    explicit TopologyGraph(int64_t n) : adj_(n) {}

    void add(int64_t i, int64_t j, int kind)
    {
        auto& ai = adj_[i];
        if(std::find(ai.begin(), ai.end(), std::make_pair(j, kind)) == ai.end()) {ai.emplace_back(j, kind);}
        auto& aj = adj_[j];
        if(std::find(aj.begin(), aj.end(), std::make_pair(i, kind)) == aj.end()) {aj.emplace_back(i, kind);}
    }

    // Topology::construct_molecules (core/Topology.hpp:280-316): one pass in
    // particle order; a particle joins the molecule of its first "bond"
    // neighbour that already has one, otherwise starts a new molecule.
    std::vector<int64_t> molecules(int bond_kind) const
    {
        const int64_t n = (int64_t)adj_.size();
        std::vector<int64_t> mol(n, -1);
        int64_t next = 0;
        for(int64_t i = 0; i < n; ++i)
        {
            for(const auto& e : adj_[i])
            {
                if(e.second != bond_kind) {continue;}
                if(mol[e.first] != -1) {mol[i] = mol[e.first]; break;}
            }
            if(mol[i] == -1) {mol[i] = next++;}
        }
        return mol;
    }

    // Topology::list_adjacent_within (core/Topology.hpp:243-260) appended to out.
    void within(int64_t i, int dist, int kind, std::vector<int64_t>& out) const
    {
        if(dist <= 0) {return;}
        std::vector<int64_t> front{i}, next;
        for(int d = 0; d < dist; ++d)
        {
            next.clear();
            for(const int64_t u : front)
            {
                for(const auto& e : adj_[u])
                {
                    if(e.second != kind) {continue;}
                    out.push_back(e.first);
                    next.push_back(e.first);
                }
            }
            std::sort(next.begin(), next.end());
            next.erase(std::unique(next.begin(), next.end()), next.end());
            front.swap(next);
        }
    }

  private:
    std::vector<std::vector<std::pair<int64_t, int>>> adj_;
};

// ExclusionList::make, topology part (core/ExclusionList.hpp:207-232): for
// every particle, itself and every particle within the given topological
// distances, sorted and unique.  Written as CSR with global offsets.
inline void exclusion_csr(const TopologyGraph& g, int64_t n,
                          const std::vector<std::pair<int, int>>& kind_within,
                          int64_t particle_offset,
                          std::vector<long long>& start, std::vector<int>& idx)
{
    std::vector<int64_t> buf;
    for(int64_t i = 0; i < n; ++i)
    {
        buf.clear();
        buf.push_back(i);
        for(const auto& kw : kind_within) {g.within(i, kw.second, kw.first, buf);}
        std::sort(buf.begin(), buf.end());
        buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
        for(const int64_t j : buf) {idx.push_back((int)(j + particle_offset));}
        start.push_back((long long)idx.size());
    }
}

}  // namespace mjg
