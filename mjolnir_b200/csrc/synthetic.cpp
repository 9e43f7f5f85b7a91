// Seeded builders of the synthetic benchmark systems (host only).  The named
// workloads are synthetic by definition; these generate their coordinates fast
// enough for million-bead batches.  No counterpart in the reference.
#include "../../include/mjolnir_b200_synthetic.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>

namespace {

// splitmix64 (Steele, Lea, Flood, "Fast splittable pseudorandom number
// generators", OOPSLA'14) as a small seeded stream
struct SplitMix {
    uint64_t s;
    explicit SplitMix(uint64_t seed) : s(seed) {}
    uint64_t next()
    {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() {return (double)(next() >> 11) * (1.0 / 9007199254740992.0);}   // [0,1)
    double normal()
    {
        double u = uniform();
        while(u <= 0.0) {u = uniform();}
        const double v = uniform();
        return std::sqrt(-2.0 * std::log(u)) * std::cos(6.283185307179586 * v);
    }
};

struct Hash {
    size_t operator()(const int64_t k) const {return (size_t)(k * 0x9E3779B97F4A7C15ull);}
};

inline int64_t key(int64_t x, int64_t y, int64_t z)
{
    return ((x + (1 << 20)) << 42) | ((y + (1 << 20)) << 21) | (z + (1 << 20));
}

}  // namespace

extern "C" MJG_SYNTH_API int mjg_synth_polymer_chains(int64_t nchains, int64_t nbeads, double bond,
                                                      double min_dist, double radius, uint64_t seed,
                                                      double* out)
{
    if(nchains <= 0 || nbeads <= 0 || !out || !(bond > 0) || !(radius > 0) || min_dist < 0) {return -1;}
    SplitMix rng(seed);
    const double cell = min_dist > 0 ? min_dist : 1.0;
    std::unordered_map<int64_t, std::vector<int64_t>, Hash> grid;
    grid.reserve((size_t)(nchains * nbeads));
    const double md2 = min_dist * min_dist;
    int64_t k = 0;
    auto cell_of = [&](const double* p, int64_t* c) {
        for(int d = 0; d < 3; ++d) {c[d] = (int64_t)std::floor(p[d] / cell);}
    };
    auto ok = [&](const double* p, int64_t skip) {
        if(p[0] * p[0] + p[1] * p[1] + p[2] * p[2] > radius * radius) {return false;}
        int64_t c[3];
        cell_of(p, c);
        for(int dx = -1; dx <= 1; ++dx)
        for(int dy = -1; dy <= 1; ++dy)
        for(int dz = -1; dz <= 1; ++dz)
        {
            auto it = grid.find(key(c[0] + dx, c[1] + dy, c[2] + dz));
            if(it == grid.end()) {continue;}
            for(const int64_t q : it->second)
            {
                if(q == skip) {continue;}
                const double ex = p[0] - out[3 * q], ey = p[1] - out[3 * q + 1], ez = p[2] - out[3 * q + 2];
                if(ex * ex + ey * ey + ez * ez < md2) {return false;}
            }
        }
        return true;
    };
    auto add = [&](const double* p) {
        out[3 * k] = p[0]; out[3 * k + 1] = p[1]; out[3 * k + 2] = p[2];
        int64_t c[3];
        cell_of(p, c);
        grid[key(c[0], c[1], c[2])].push_back(k);
        ++k;
    };
    auto remove_last = [&]() {
        --k;
        int64_t c[3];
        cell_of(out + 3 * k, c);
        grid[key(c[0], c[1], c[2])].pop_back();   // beads leave in reverse order of arrival
    };
    for(int64_t ch = 0; ch < nchains; ++ch)
    {
        const int64_t first = k;
        bool done = false;
        for(int restart = 0; restart < 1000 && !done; ++restart)
        {
            while(k > first) {remove_last();}
            int tries = 0;
            for(;;)
            {
                double p[3] = {(2 * rng.uniform() - 1) * radius, (2 * rng.uniform() - 1) * radius,
                               (2 * rng.uniform() - 1) * radius};
                if(ok(p, -1)) {add(p); break;}
                if(++tries > 100000) {return -2;}
            }
            done = true;
            for(int64_t b = 1; b < nbeads && done; ++b)
            {
                const double* prev = out + 3 * (k - 1);
                bool placed = false;
                for(int t = 0; t < 200 && !placed; ++t)
                {
                    double d[3] = {rng.normal(), rng.normal(), rng.normal()};
                    const double nrm = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                    if(!(nrm > 0)) {continue;}
                    double p[3] = {prev[0] + bond * d[0] / nrm, prev[1] + bond * d[1] / nrm,
                                   prev[2] + bond * d[2] / nrm};
                    if(ok(p, k - 1)) {add(p); placed = true;}
                }
                if(!placed) {done = false;}   // dead end: grow this chain again
            }
        }
        if(!done) {return -3;}
    }
    return 0;
}

// Uniform positions in [0, L)^3 with every pair at least min_dist apart under
// the minimum image (random sequential addition with redraws).
extern "C" MJG_SYNTH_API int mjg_synth_uniform_fluid(int64_t n, double L, double min_dist, uint64_t seed,
                                                     double* out)
{
    if(n <= 0 || !(L > 0) || !out || min_dist < 0) {return -1;}
    SplitMix rng(seed);
    const int64_t nc = std::max<int64_t>(1, (int64_t)std::floor(L / (min_dist > 0 ? min_dist : L)));
    const double w = L / (double)nc;
    std::unordered_map<int64_t, std::vector<int64_t>, Hash> grid;
    grid.reserve((size_t)n);
    const double md2 = min_dist * min_dist;
    for(int64_t k = 0; k < n; ++k)
    {
        for(int tries = 0;; ++tries)
        {
            if(tries > 1000000) {return -2;}
            double p[3] = {rng.uniform() * L, rng.uniform() * L, rng.uniform() * L};
            int64_t c[3];
            for(int d = 0; d < 3; ++d) {c[d] = std::min<int64_t>(nc - 1, (int64_t)(p[d] / w));}
            bool good = true;
            if(min_dist > 0)
            {
                for(int dx = -1; dx <= 1 && good; ++dx)
                for(int dy = -1; dy <= 1 && good; ++dy)
                for(int dz = -1; dz <= 1 && good; ++dz)
                {
                    const int64_t x = ((c[0] + dx) % nc + nc) % nc, y = ((c[1] + dy) % nc + nc) % nc,
                                  z = ((c[2] + dz) % nc + nc) % nc;
                    auto it = grid.find(key(x, y, z));
                    if(it == grid.end()) {continue;}
                    for(const int64_t q : it->second)
                    {
                        double e[3];
                        for(int d = 0; d < 3; ++d)
                        {
                            e[d] = p[d] - out[3 * q + d];
                            if(e[d] < -L / 2) {e[d] += L;} else if(e[d] >= L / 2) {e[d] -= L;}
                        }
                        if(e[0] * e[0] + e[1] * e[1] + e[2] * e[2] < md2) {good = false; break;}
                    }
                }
            }
            if(!good) {continue;}
            out[3 * k] = p[0]; out[3 * k + 1] = p[1]; out[3 * k + 2] = p[2];
            grid[key(c[0], c[1], c[2])].push_back(k);
            break;
        }
    }
    return 0;
}
