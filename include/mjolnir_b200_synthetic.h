/*
 * Seeded synthetic-system builders shipped in libmjolnir_b200.so (host code,
 * no GPU needed).  They produce the coordinates of the benchmark workloads;
 * they have no counterpart in the reference, whose inputs are TOML files.
 * Return 0 on success, a negative value when the parameters are invalid or
 * the packing cannot be completed.
 */
#ifndef MJOLNIR_B200_SYNTHETIC_H
#define MJOLNIR_B200_SYNTHETIC_H
#include <stdint.h>

#if defined(__GNUC__)
#define MJG_SYNTH_API __attribute__((visibility("default")))
#else
#define MJG_SYNTH_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* nchains random-walk chains of nbeads beads, bond-long steps in seed-drawn
 * directions, every bead at least min_dist from every bead other than the one
 * it is bonded to, all inside a sphere of `radius` around the origin.
 * out[3 nchains nbeads]. */
MJG_SYNTH_API int mjg_synth_polymer_chains(int64_t nchains, int64_t nbeads, double bond,
                                           double min_dist, double radius, uint64_t seed,
                                           double* out);

/* n uniform positions in the periodic cube [0, L)^3, pairwise at least
 * min_dist apart under the minimum image.  out[3 n]. */
MJG_SYNTH_API int mjg_synth_uniform_fluid(int64_t n, double L, double min_dist, uint64_t seed,
                                          double* out);

#ifdef __cplusplus
}
#endif
#endif
