/*
 * mjolnir_b200 -- C ABI of the B200 implementation of Mjolnir's per-step hot
 * path: cell-list / Verlet-list rebuild, ExcludedVolume, DebyeHuckel and
 * LennardJones pair forces and energies, harmonic bonds and angles, cosine
 * dihedrals, and the BAOAB Langevin (or velocity Verlet) update.
 *
 * Plain pointers and sizes only.  Every call returns MJG_OK (0) or a negative
 * MJG_E* code, and mjg_last_error() then describes the failure; no C++
 * exception crosses this boundary.  Host arrays are owned by the caller and
 * are only read (or written) during the call.  Device memory is owned by the
 * context.  A context is used by one host thread at a time.
 *
 * Mjolnir has no C ABI and no plugin loader: the GPU path replaces the C++
 * virtual interfaces named beside each entry point.  Citations are
 * path:line inside the Mjolnir source tree (v1.31.0).
 *
 * Indices are 0-based particle indices local to their system.  Units are
 * kcal/mol and angstrom: kB, the vacuum permittivity and the volume factor
 * are those input/read_units.hpp:32-91 derives for these units.
 */
#ifndef MJOLNIR_B200_H
#define MJOLNIR_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define MJG_API __attribute__((visibility("default")))
#else
#define MJG_API
#endif

typedef struct mjg_context mjg_context;

enum {
    MJG_OK = 0,
    MJG_EINVAL = -1,      /* bad argument                                   */
    MJG_ECUDA = -2,       /* a CUDA call failed                             */
    MJG_ESTATE = -3,      /* call not allowed in the current state          */
    MJG_ENOMEM = -4,      /* device memory exhausted                        */
    MJG_EOVERFLOW = -5,   /* a force left the fixed-point range             */
    MJG_ENONFINITE = -6   /* non-finite positions or forces (blown up)      */
};
enum { MJG_PRECISION_FP64 = 0, MJG_PRECISION_MIXED = 1 };
enum { MJG_UNLIMITED = 0, MJG_PERIODIC_CUBOID = 1 };
enum { MJG_TERM_BOND = 0, MJG_TERM_ANGLE = 1, MJG_TERM_DIHEDRAL = 2,
       MJG_TERM_EXV = 3, MJG_TERM_DH = 4, MJG_TERM_LJ = 5 };
enum { MJG_IGNORE_NOTHING = 0, MJG_IGNORE_SELF = 1, MJG_IGNORE_OTHERS = 2 };
enum { MJG_BAOAB = 0, MJG_VELOCITY_VERLET = 1, MJG_UNDERDAMPED_LANGEVIN = 2, MJG_GJF_LANGEVIN = 3,
       MJG_GBAOAB_LANGEVIN = 4 };

/* ---------------------------------------------------------------- context */

/* A context owns one arena on one device: every committed system lives in
 * it, and mjg_step advances all of them in the same kernels.
 * precision: MJG_PRECISION_FP64 (the reference's arithmetic) or
 * MJG_PRECISION_MIXED (FP32 pair potentials, FP64 state, forces summed in
 * 64-bit fixed point).  No counterpart in the reference (its parallelism is
 * OpenMP inside one process, mjolnir/omp/*). */
MJG_API int  mjg_context_create(int device, int precision, mjg_context** out);
MJG_API void mjg_context_destroy(mjg_context* ctx);
MJG_API const char* mjg_last_error(const mjg_context* ctx);
/* 1: capture one MD step as a CUDA graph and replay it (default 1). */
MJG_API int  mjg_context_set_graphs(mjg_context* ctx, int enable);
/* Options: the per-step work of mjg_step is also checked for list overflow
 * and rolled back when it happens (default 1). */
MJG_API int  mjg_context_set_rollback(mjg_context* ctx, int enable);
/* Reserves the page-locked host buffers that commits pack into for an
 * arena of up to `particles` particles (about 450 bytes per particle), so
 * that a server which fills its arena over many commits does not page-lock
 * memory again and again while it serves.  Optional; buffers still grow
 * when a commit needs more. */
MJG_API int  mjg_context_reserve(mjg_context* ctx, int64_t particles);

/* ---------------------------------------------------------------- systems */

/* System<traits>(num_particles, boundary) with its particles
 * (core/System.hpp:41-52; input/read_system.hpp:93-290).  lower/upper are
 * the periodic box (ignored for MJG_UNLIMITED).  pos/vel/mass: [3n], [3n], [n].
 * Positions are wrapped into the box (System::initialize, core/System.hpp:58-67).
 * Returns the system id through *sys_id. */
MJG_API int mjg_system_create(mjg_context* ctx, int64_t n, int boundary,
                      const double* lower, const double* upper,
                      const double* pos, const double* vel, const double* mass,
                      int* sys_id);
/* system.attributes temperature [K] and ionic_strength [mol/L]
 * (core/System.hpp:151-156).  Temperature 0 runs without thermal noise (a
 * system with DebyeHuckel needs a positive temperature for its Debye length,
 * checked at mjg_commit); the ionic strength must be positive. */
MJG_API int mjg_system_set_attributes(mjg_context* ctx, int sys, double temperature,
                              double ionic_strength);
/* Topology::add_connection for m pairs of the connection kind `kind`
 * (core/Topology.hpp:165-195), e.g. a force-free "bond" chain
 * (forcefield/local/DummyInteraction.hpp). */
MJG_API int mjg_system_add_connections(mjg_context* ctx, int sys, const char* kind,
                               int64_t m, const int64_t* pairs);
/* Changes a system's temperature at any time: the Langevin noise coefficients
 * of its particles take the new value from the next step on, as
 * BAOABLangevinIntegrator::update does after SimulatedAnnealingSimulator sets
 * the temperature attribute (core/SimulatedAnnealingSimulator.hpp:144-154,
 * core/BAOABLangevinIntegrator.hpp:47-58).  DebyeHuckel keeps the Debye
 * length of the committed temperature, as the reference's annealing does. */
MJG_API int mjg_system_set_temperature(mjg_context* ctx, int sys, double temperature);
/* Sets the integrator's step counter of a system before its first commit
 * (default 0).  The Langevin noise of particle i at step t is Philox keyed by
 * (seed, i, t), so a system restored from a checkpoint with the step it had
 * continues the same noise stream.  The reference keeps its mt19937 state in
 * the checkpoint's _rng.msg instead (core/MsgPackSaver.hpp:66-87). */
MJG_API int mjg_system_set_step(mjg_context* ctx, int sys, uint64_t step);
/* Freezes (1) or releases (0) a system: while frozen it does not advance in
 * mjg_step and its forces, energies and state stay as they are (its terms are
 * not evaluated), so a finished job can wait in the arena until the next
 * mjg_commit removes it.  Takes effect between mjg_step calls.  No
 * counterpart in the reference (one simulation per process). */
MJG_API int mjg_system_freeze(mjg_context* ctx, int sys, int frozen);
/* Removes a system; its device state is freed at the next mjg_commit. */
MJG_API int mjg_system_remove(mjg_context* ctx, int sys);

/* ------------------------------------------------- global pair interactions
 * GlobalPairInteraction<traits, Potential> (core/GlobalInteractionBase.hpp
 * :20-36; forcefield/global/GlobalPairInteraction.hpp:26-136) with a
 * CellList spatial partition of relative margin `margin`
 * (input/read_spatial_partition.hpp:62-76; core/PeriodicGridCellList.hpp,
 * core/UnlimitedGridCellList.hpp).  idx[np] lists the participants in input
 * order; the last one leads no list (ParameterList leading_participants). */

/* ExcludedVolumePotential(cutoff_ratio, epsilon) + ExcludedVolumeParameterList
 * (forcefield/global/ExcludedVolumePotential.hpp:26-133,139-282). */
MJG_API int mjg_exv_set(mjg_context* ctx, int sys, double epsilon, double cutoff_ratio,
                double margin, int64_t np, const int64_t* idx, const double* radius);
/* DebyeHuckelPotential(cutoff_ratio) + DebyeHuckelParameterList
 * (forcefield/global/DebyeHuckelPotential.hpp:17-186,196-353); uses the
 * system's temperature and ionic_strength. */
MJG_API int mjg_dh_set(mjg_context* ctx, int sys, double cutoff_ratio, double margin,
               int64_t np, const int64_t* idx, const double* charge);
/* LennardJonesPotential(cutoff_ratio) + LorentzBerthelotRule
 * (forcefield/global/LennardJonesPotential.hpp:15-110, ParameterList.hpp:185-329). */
MJG_API int mjg_lj_set(mjg_context* ctx, int sys, double cutoff_ratio, double margin,
               int64_t np, const int64_t* idx, const double* sigma, const double* epsilon);
/* The first global term with another potential of the ExcludedVolume
 * family, by the reference's input name: "InversePower"
 * (forcefield/global/InversePowerPotential.hpp; per-particle radius in p0,
 * sigma_ij = r_i + r_j, E = eps ((sigma/r)^n - rc^-n), exponent `power`) or
 * "HardCoreExcludedVolume" (HardCoreExcludedVolumePotential.hpp; per-particle
 * soft_shell_thickness in p0 and core_radius in p1, sigma_ij and R_ij the
 * sums, E = eps ((sigma / (r - R))^12 - rc^-12)).  Both run through the
 * generic pair loop (GlobalPairInteraction.hpp:148-213). */
MJG_API int mjg_exv_family_set(mjg_context* ctx, int sys, const char* potential, double epsilon,
                               double cutoff_ratio, int power, double margin, int64_t np,
                               const int64_t* idx, const double* p0, const double* p1);
/* The third global term with any potential of the Lennard-Jones family, by
 * the name the reference's input uses: "LennardJones" (as mjg_lj_set),
 * "WCA" (forcefield/global/WCAPotential.hpp; its cutoff is fixed at
 * 2^(1/6) sigma and cutoff_ratio is ignored, as input/read_global_potential.hpp
 * warns), "LennardJonesAttractive" (LennardJonesAttractivePotential.hpp) or
 * "UniformLennardJones" (UniformLennardJonesPotential.hpp; every participant
 * must carry the same sigma and epsilon).  The last three run through the
 * generic GlobalPairInteraction loop (GlobalPairInteraction.hpp:148-213) with
 * the Lorentz-Berthelot rule (ParameterList.hpp:240-251). */
MJG_API int mjg_pair_set(mjg_context* ctx, int sys, const char* potential, double cutoff_ratio,
                         double margin, int64_t np, const int64_t* idx, const double* sigma,
                         const double* epsilon);
/* The ignore rules of one global term: ignore.molecule and
 * ignore.particles_within (input/read_global_potential.hpp:29-90,168-190;
 * core/ExclusionList.hpp:56-234).  kinds[k] / within[k] for nk connection
 * kinds.  Default: ignore nothing. */
MJG_API int mjg_ignore_set(mjg_context* ctx, int sys, int term, int ignore_molecule,
                   int nk, const char* const* kinds, const int32_t* within);

/* ------------------------------------------------------ local interactions
 * LocalInteractionBase<traits> (core/LocalInteractionBase.hpp:24-40);
 * `topology` is the connection kind written to the topology
 * (write_topology), "none" for no edges. */

/* BondLengthInteraction<HarmonicPotential> (BondLengthInteraction.hpp:126-148,
 * HarmonicPotential.hpp:11-52; V = k (r - v0)^2). idx[2m]. */
MJG_API int mjg_bonds_set(mjg_context* ctx, int sys, const char* topology, int64_t m,
                  const int64_t* idx, const double* k, const double* v0);
/* BondAngleInteraction<HarmonicPotential> (BondAngleInteraction.hpp:129-188). idx[3m]. */
MJG_API int mjg_angles_set(mjg_context* ctx, int sys, const char* topology, int64_t m,
                   const int64_t* idx, const double* k, const double* v0);
/* DihedralAngleInteraction<CosinePotential> (DihedralAngleInteraction.hpp
 * :157-227, CosinePotential.hpp:13-58; V = k (1 + cos(n (phi - v0)))). idx[4m]. */
MJG_API int mjg_dihedrals_set(mjg_context* ctx, int sys, const char* topology, int64_t m,
                      const int64_t* idx, const double* k, const int32_t* n,
                      const double* v0);

/* -------------------------------------------------------------- integrator
 * BAOABLangevinIntegrator(dt, gammas) (core/BAOABLangevinIntegrator.hpp:34-99;
 * input/read_integrator.hpp:120-187), VelocityVerletIntegrator(dt)
 * (core/VelocityVerletIntegrator.hpp) or UnderdampedLangevinIntegrator(dt,
 * gammas) (core/UnderdampedLangevinIntegrator.hpp; its acceleration with noise
 * is carried from step to step, across commits and rollbacks; replacing a
 * system's positions starts it again as Integrator::initialize does) or
 * GJFNVTLangevinIntegrator(dt, alphas) (core/GJFNVTLangevinIntegrator.hpp,
 * "G-JFLangevin"; input/read_integrator.hpp:242-300) or
 * gBAOABLangevinIntegrator(dt, gammas) (core/gBAOABLangevinIntegrator.hpp,
 * "g-BAOABLangevin"; :189-239) without constraints: BAOAB whose two half
 * drifts each move the position.
 * gamma[n]: the friction gammas, or the G-JF alphas (ignored for Verlet).  The Langevin noise is Philox4x32-10 keyed
 * by `seed` and counted by (particle, step), in place of the reference's
 * mt19937 stream (core/RandomNumberGenerator.hpp:13-86); the underdamped
 * closing of step t draws counter t + 1, its initialisation the current
 * step, so a resumed system repeats the acceleration it had. */
MJG_API int mjg_integrator_set(mjg_context* ctx, int sys, int kind, double dt,
                       const double* gamma, uint64_t seed);

/* ------------------------------------------------------------- execution */

/* Packs every live system into device memory, builds the topology,
 * exclusion lists, cell lists and Verlet lists, and evaluates the first
 * forces (ForceField::initialize, core/ForceField.hpp:47-63, and
 * Integrator::initialize, core/BAOABLangevinIntegrator.hpp:135-168).
 * Systems already resident keep their positions, velocities, forces and
 * noise counters.  Call again after adding or removing systems. */
MJG_API int mjg_commit(mjg_context* ctx);
/* nsteps integrator steps of every committed system
 * (BAOABLangevinIntegrator::step, core/BAOABLangevinIntegrator.hpp:170-240,
 * called by MolecularDynamicsSimulator::step, core/MolecularDynamicsSimulator.hpp:83-102). */
MJG_API int mjg_step(mjg_context* ctx, int64_t nsteps);
/* Waits for the context's stream. */
MJG_API int mjg_synchronize(mjg_context* ctx);
/* Rebuilds every Verlet list at the current positions. */
MJG_API int mjg_rebuild(mjg_context* ctx);

/* State of one system in host layout [3n] (NULL to skip an array).
 * mjg_set_state replaces positions and/or velocities (wrapped into the box)
 * and marks the lists for a rebuild. */
MJG_API int mjg_get_state(mjg_context* ctx, int sys, double* pos, double* vel, double* force);
MJG_API int mjg_set_state(mjg_context* ctx, int sys, const double* pos, const double* vel);
/* Same for all committed systems at once, concatenated in commit order. */
MJG_API int mjg_get_state_all(mjg_context* ctx, double* pos, double* vel);
MJG_API int mjg_set_state_all(mjg_context* ctx, const double* pos, const double* vel);

/* Energies of every term at the current positions, out[6] indexed by
 * MJG_TERM_* (ForceField::calc_energy / format_energy, core/ForceField.hpp:123-160). */
MJG_API int mjg_energies(mjg_context* ctx, int sys, double* out);
/* Forces [3n] and energy of a single term at the current positions, without
 * disturbing the integrator's force array (GlobalInteractionBase /
 * LocalInteractionBase::calc_force_and_energy). */
MJG_API int mjg_term_force(mjg_context* ctx, int sys, int term, double* force, double* energy);
/* The half Verlet list of a global term as it was last built, as (i, j)
 * pairs with i < j sorted by i then j -- the content of
 * SpatialPartition::neighbors() (core/NeighborList.hpp:151-266).  Writes at
 * most cap pairs to pairs[2 cap] and the total to *count. */
MJG_API int mjg_neighbors(mjg_context* ctx, int sys, int term, int64_t* pairs,
                  int64_t cap, int64_t* count);
/* Number of interacting pairs (i < j inside the potential's own cutoff) of a
 * global term at the current positions, for one system or all (sys = -1):
 * the margin-free pair count P_cut of the pair kernel's roofline.  No
 * counterpart in the reference. */
MJG_API int mjg_pair_count(mjg_context* ctx, int sys, int term, int64_t* count);
/* The CUDA stream (cudaStream_t) all of the context's work is enqueued on,
 * for callers that record events or order their own work against it. */
MJG_API int mjg_context_get_stream(mjg_context* ctx, void** stream);
/* Average duration in milliseconds of one launch of a term's force kernel
 * (pair kernel for MJG_TERM_EXV/DH/LJ, bonded kernel otherwise) on the
 * current lists over `reps` launches, each timed with CUDA events on the
 * context's stream after a 256 MiB write has evicted L2 and a 256 MiB read
 * of another buffer has replaced the written lines with clean ones; the
 * integrator's forces are not touched.  Allocates and frees the two
 * buffers. */
MJG_API int mjg_time_kernel(mjg_context* ctx, int term, int reps, double* ms_per_launch);
/* Performance knobs of a global term (they change no result in the mixed
 * form, whose force sums are exact and order independent):
 * threads cooperating on one particle's list in the pair kernel (1, 2, 4, 8,
 * 16 or 32; re-lays out and rebuilds the lists; schedules 2 and 3 run as
 * schedule 0 at 32), and the relative Verlet margin
 * of every system that has the term (re-commits: new cell grids, new lists,
 * state kept).  The reference fixes the margin in its input
 * (input/read_spatial_partition.hpp:62-76). */
MJG_API int mjg_set_threads_per_particle(mjg_context* ctx, int term, int tpp);
MJG_API int mjg_get_threads_per_particle(mjg_context* ctx, int term, int* tpp);
MJG_API int mjg_set_margin(mjg_context* ctx, int term, double margin);
/* Partners a thread requests per batch in a global term's force launch (1, 2
 * or 4): deeper batches keep more loads in flight per thread at the cost of
 * registers.  A launch-shape knob like the threads per particle; it changes
 * no result.  No counterpart in the reference. */
MJG_API int mjg_set_pair_unroll(mjg_context* ctx, int term, int unroll);
MJG_API int mjg_get_pair_unroll(mjg_context* ctx, int term, int* unroll);
/* Schedule of a global term's force launch: 0 = one particle per group of
 * threads-per-particle threads; 1 (mixed form only) = warp-balanced, a warp
 * splits the combined lists of its 32 particles evenly over its lanes and adds
 * each partial sum with integer atomics (exact, so the forces are identical);
 * 2 = one thread per particle reading its list in blocks of
 * threads-per-particle words with vector loads (with threads-per-particle 1
 * it is schedule 0); 3 = as 2, with the threads of each 256-particle block
 * handed its particles in order of list length; 4 = as 0, with the thread
 * groups of each block handed its particles in order of list length; 5 = as
 * 0 on lists stored particle by particle (contiguous), each particle's list
 * requested into L2 by one bulk prefetch as its group starts (switching to or
 * from 5 rebuilds every list of the term).  No counterpart in the reference. */
MJG_API int mjg_set_pair_schedule(mjg_context* ctx, int term, int schedule);
MJG_API int mjg_get_pair_schedule(mjg_context* ctx, int term, int* schedule);
/* Half Verlet lists for a global term (mixed form only; MJG_EINVAL in the
 * FP64 form): a pair is stored in the list of its lower slot alone, and the
 * force launch adds the pair's negated fixed-point force to the partner with
 * integer atomics -- the same integer sums as the full lists, so forces and
 * trajectories are identical bit for bit, with half the list words and pair
 * evaluations for the atomics of the partners' shares.  Switching rebuilds
 * every list of the term.  mjg_neighbors reports the same pairs either way.
 * The reference's own lists are half lists (core/NeighborList.hpp:151-266,
 * pairs j > i); its force loop adds f to i and subtracts it from j
 * (GlobalPairInteraction.hpp:148-213). */
MJG_API int mjg_set_half_lists(mjg_context* ctx, int term, int on);
MJG_API int mjg_get_half_lists(mjg_context* ctx, int term, int* on);
/* Lanes per particle of a global term's list build (4, 8, 16 or 32): fewer
 * lanes build several lists per warp at once, which pays when a particle has
 * few candidates in its 27 neighbouring cells.  Unless set here, each commit
 * picks it from the candidates an even filling of the grids would give
 * (below 12: 8, below 64: 16, else 32).  The lists are the same in every
 * case.  No counterpart in the reference. */
MJG_API int mjg_set_build_lanes(mjg_context* ctx, int term, int lanes);
MJG_API int mjg_get_build_lanes(mjg_context* ctx, int term, int* lanes);
/* Sets the per-particle neighbour capacity of a global term's lists.  A
 * capacity below what a later rebuild needs is detected on the device, the
 * current mjg_step chunk is rolled back, the lists grow and the chunk runs
 * again (with rollback enabled); used to test that path.  No counterpart in
 * the reference, whose lists are growable std::vectors. */
MJG_API int mjg_set_list_capacity(mjg_context* ctx, int term, int cap);
/* Number of list rebuilds of a term since commit (reduce_margin rebuilds). */
MJG_API int mjg_rebuild_count(mjg_context* ctx, int sys, int term, int64_t* count);
/* Number of integrator steps taken by a system since it was created. */
MJG_API int mjg_step_count(mjg_context* ctx, int sys, int64_t* steps);
/* Number of molecules of a system: the groups of particles joined by "bond"
 * connections (Topology::construct_molecules, core/Topology.hpp:280-316;
 * Topology::number_of_molecules, :118), as the DCD header records them. */
MJG_API int mjg_molecule_count(mjg_context* ctx, int sys, int64_t* count);

/* Number of particles of all committed systems, and of one system. */
MJG_API int mjg_particle_count(mjg_context* ctx, int sys, int64_t* n);
/* Bytes of device memory the context holds. */
MJG_API int mjg_device_bytes(mjg_context* ctx, int64_t* bytes);
/* Kernel launches issued since the context was created (graph replays count
 * each kernel node). */
MJG_API int mjg_launch_count(mjg_context* ctx, int64_t* launches);

/* ------------------------------------------------- allocation-free variant
 * No counterpart in the reference.  For callers that may not allocate device
 * memory themselves -- a host framework that owns every device allocation
 * through its own pool, or an embedding that forbids cudaMalloc once it has
 * started -- and so cannot create a context (mjg_commit allocates its arena).
 *
 * ExcludedVolume forces and energy of one system whose arrays the caller
 * already holds in device memory: pos [3n] and radius [n] in, force [3n] and
 * energy [1] out (both overwritten), enqueued on `stream` (a cudaStream_t;
 * NULL for the default stream).  Every particle takes part, no pair is
 * excluded, FP64 arithmetic -- the quantity mjg_term_force gives for
 * MJG_TERM_EXV of a system without ignore rules.  lower/upper (host, 3 each)
 * give the periodic box for MJG_PERIODIC_CUBOID; positions may lie outside it
 * by up to a quarter of its width on each side (cells wrap, and each
 * displacement takes one periodic shift, as the reference's adjust_direction);
 * they are ignored for MJG_UNLIMITED.
 *
 * The call allocates nothing: its cell list lives in one fixed device array of
 * about 1 MiB that every GPU loading the library keeps until the process
 * exits, which limits n to 65536 (larger n returns MJG_EINVAL and prints the
 * limit).  The first call in a CUDA context (the first on a device, and the
 * first after a device reset) looks up that array's device address; make it
 * before any stream capture.  All calls share the array:
 * calls that overlap on the GPU (other streams, other threads) race and give
 * wrong results, so serialise them. */
MJG_API int mjg_exv_force_noalloc(int64_t n, int boundary, const double* lower,
                                  const double* upper, const double* pos, const double* radius,
                                  double epsilon, double cutoff_ratio, double* force,
                                  double* energy, void* stream);

#ifdef __cplusplus
}
#endif
#endif
