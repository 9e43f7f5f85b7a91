/*
 * Flat, C-layout description of one Mjolnir system, shared by the two CPU
 * checkers under oracle/ (TEST INFRASTRUCTURE, never the product path):
 *
 *   - oracle/ref_driver.cpp  builds the *reference's own* objects
 *     (mjolnir::System, ForceField, GlobalPairInteraction, BAOAB ...) from it,
 *     compiled from the unmodified reference headers into oracle/_ref/;
 *   - oracle/oracle.c        is a plain-C restatement of the same algorithms.
 *
 * Units are the reference's kcal/mol + angstrom system (input/read_units.hpp:32-91).
 * Index arrays are int64 particle indices (the reference's std::size_t).
 */
#ifndef MJOLNIR_ORACLE_SPEC_H
#define MJOLNIR_ORACLE_SPEC_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_UNLIMITED = 0, ORC_PERIODIC = 1 };
enum { ORC_BAOAB = 0, ORC_VV = 1, ORC_UNDERDAMPED = 2, ORC_GJF = 3, ORC_GBAOAB = 4 };
enum { ORC_IGNORE_NOTHING = 0, ORC_IGNORE_SELF = 1, ORC_IGNORE_OTHERS = 2 };
/* potential of the first global term (ExcludedVolume family) */
enum { ORC_EXV = 0, ORC_INVERSE_POWER = 1, ORC_HARD_CORE_EXV = 2 };
/* potential of the third global term (Lennard-Jones family) */
enum { ORC_LJ = 0, ORC_WCA = 1, ORC_LJ_ATTRACTIVE = 2, ORC_LJ_UNIFORM = 3 };
enum { ORC_TERM_BOND = 0, ORC_TERM_ANGLE = 1, ORC_TERM_DIHEDRAL = 2,
       ORC_TERM_EXV = 3, ORC_TERM_DH = 4, ORC_TERM_LJ = 5, ORC_NTERMS = 6 };

typedef struct orc_spec
{
    int64_t n;
    int32_t boundary;            /* ORC_UNLIMITED / ORC_PERIODIC            */
    int32_t single_molecule;     /* 1: add a "bond" chain 0-1-2-... through a
                                    force-free Dummy interaction so that a
                                    bond-free fluid is one molecule          */
    double lower[3], upper[3];   /* periodic box                            */
    const double* pos;           /* [3n]                                    */
    const double* vel;           /* [3n]                                    */
    const double* mass;          /* [n]                                     */
    double temperature;          /* K                                       */
    double ionic_strength;       /* mol/L                                   */

    /* global pair terms; ignore rules are shared by all three            */
    int32_t ignore_molecule;     /* ORC_IGNORE_*                            */
    int32_t ignore_bond_within;  /* ignore.particles_within.bond (0: none)  */

    int32_t exv_on;  double exv_eps, exv_cutoff, exv_margin;
    int64_t exv_n;   const int64_t* exv_idx; const double* exv_radius;
    int32_t exv_kind;            /* ORC_EXV / ORC_INVERSE_POWER / ORC_HARD_CORE_EXV */
    int32_t exv_power;           /* InversePower n                          */
    const double* exv_core;      /* HardCoreExcludedVolume core_radius (exv_radius: soft_shell_thickness) */

    int32_t dh_on;   double dh_cutoff, dh_margin;
    int64_t dh_n;    const int64_t* dh_idx;  const double* dh_charge;

    int32_t lj_on;   double lj_cutoff, lj_margin;
    int64_t lj_n;    const int64_t* lj_idx;  const double* lj_sigma;
    const double* lj_eps;
    int32_t lj_kind;             /* ORC_LJ / ORC_WCA / ORC_LJ_ATTRACTIVE / ORC_LJ_UNIFORM */

    /* local terms (BondLength topology "bond"; angle/dihedral "none")     */
    int64_t nbond;   const int64_t* bond_idx;  const double* bond_k;
    const double* bond_v0;
    int64_t nangle;  const int64_t* angle_idx; const double* angle_k;
    const double* angle_v0;
    int64_t ndihd;   const int64_t* dihd_idx;  const double* dihd_k;
    const int32_t* dihd_n; const double* dihd_v0;

    /* integrator */
    int32_t integrator;          /* ORC_BAOAB / _VV / _UNDERDAMPED / _GJF / _GBAOAB */
    double  dt;
    const double* gamma;         /* [n] friction (G-JF: alpha)              */
    uint64_t seed;
} orc_spec;

#ifdef __cplusplus
}
#endif
#endif
