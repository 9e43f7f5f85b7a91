"""Plain description of one Mjolnir system and seeded synthetic builders.

A :class:`SystemDesc` carries exactly what the reference reads from its TOML
input for the per-step hot path (``[[systems]]`` particles and attributes,
``[[forcefields.global]]`` ExcludedVolume / DebyeHuckel / LennardJones with
their ``ignore`` rules and ``spatial_partition``, ``[[forcefields.local]]``
BondLength / BondAngle / DihedralAngle, and the BAOAB ``[simulator]``
settings; input/read_system.hpp:93-290, input/read_global_potential.hpp,
input/read_local_interaction.hpp, input/read_integrator.hpp:120-187).

Units are kcal/mol and angstrom throughout (input/read_units.hpp:32-91).
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

KB_KCAL = 1.38064852e-23 * (1.0 / 4.184 / 1000.0) * 6.022140857e23  # kB in kcal/mol/K


@dataclasses.dataclass
class PairTerm:
    """One ``[[forcefields.global]]`` pair interaction."""
    kind: str                          # "ExcludedVolume" | "InversePower" | "HardCoreExcludedVolume"
                                       # (the first global term, SystemDesc.exv) | "DebyeHuckel" |
                                       # "LennardJones" | "WCA" | "LennardJonesAttractive" |
                                       # "UniformLennardJones" (the third, SystemDesc.lj)
    idx: np.ndarray                    # participant particle indices (input order)
    param0: np.ndarray                 # radius | charge | sigma (HardCore: soft_shell_thickness)
    param1: Optional[np.ndarray] = None  # LJ-family epsilon | HardCore core_radius
    cutoff: float = 2.0                # relative cutoff (potential default)
    margin: float = 0.5                # relative Verlet skin of the cell list
    epsilon: float = 0.2               # ExcludedVolume / InversePower / HardCoreExcludedVolume epsilon
    exponent: int = 12                 # InversePower n
    # this term's own ``ignore`` table; None falls back to the system-wide rule
    ignore_molecule: Optional[str] = None       # "Nothing" | "Self" | "Others"
    ignore_within: Optional[dict] = None        # {connection kind: topological distance}


@dataclasses.dataclass
class SystemDesc:
    pos: np.ndarray                    # (n, 3) float64
    vel: np.ndarray                    # (n, 3) float64
    mass: np.ndarray                   # (n,)
    boundary: str = "Unlimited"        # "Unlimited" | "PeriodicCuboid"
    lower: tuple = (0.0, 0.0, 0.0)
    upper: tuple = (0.0, 0.0, 0.0)
    temperature: float = 300.0
    ionic_strength: float = 0.1
    exv: Optional[PairTerm] = None
    dh: Optional[PairTerm] = None
    lj: Optional[PairTerm] = None
    ignore_molecule: str = "Nothing"   # "Nothing" | "Self" | "Others"
    ignore_bond_within: int = 0        # ignore.particles_within.bond
    single_molecule: bool = False      # fluids: one "bond"-chain molecule
    bonds: Optional[tuple] = None      # (idx (m,2) int64, k (m,), v0 (m,))
    angles: Optional[tuple] = None     # (idx (m,3), k, v0)
    dihedrals: Optional[tuple] = None  # (idx (m,4), k, n int32, v0)
    bond_topology: str = "bond"        # connection kind each local term writes
    angle_topology: str = "none"
    dihedral_topology: str = "none"
    integrator: str = "BAOAB"          # "BAOAB" | "VelocityVerlet" | "UnderdampedLangevin" | "G-JFLangevin"
                                       # | "g-BAOABLangevin"
    dt: float = 0.01
    gamma: Optional[np.ndarray] = None # friction per particle (G-JFLangevin: its alpha)
    seed: int = 12345
    start_step: int = 0                # noise step counter to resume from (checkpoints)

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])

    @property
    def periodic(self) -> bool:
        return self.boundary == "PeriodicCuboid"

    def pair_terms(self):
        return [t for t in (self.exv, self.dh, self.lj) if t is not None]

    def copy(self) -> "SystemDesc":
        return dataclasses.replace(self, pos=self.pos.copy(), vel=self.vel.copy())


# --------------------------------------------------------------------------
# seeded synthetic systems (the named workloads are synthetic: no dataset)
# --------------------------------------------------------------------------

def maxwell_boltzmann(rng: np.random.Generator, mass: np.ndarray, kT: float) -> np.ndarray:
    return rng.standard_normal((mass.shape[0], 3)) * np.sqrt(kT / mass)[:, None]


def lj_fluid(n: int = 4096, density: float = 0.8, jitter: float = 0.05,
             cutoff: float = 2.5, margin: float = 0.5, dt: float = 0.005,
             gamma: float = 1.0, seed: int = 1) -> SystemDesc:
    """Lennard-Jones fluid on a jittered simple-cubic lattice (sigma = eps = 1),
    cubic periodic box L = (n/density)^(1/3), kT = 1 (temperature 1/kB)."""
    rng = np.random.default_rng(seed)
    m = round(n ** (1.0 / 3.0))
    if m ** 3 != n:
        raise ValueError("lj_fluid needs a cubic particle count")
    L = (n / density) ** (1.0 / 3.0)
    a = L / m
    g = np.arange(m, dtype=np.float64)
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    pos = (np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1) + 0.5) * a
    pos += rng.uniform(-jitter, jitter, size=pos.shape)
    mass = np.ones(n)
    T = 1.0 / KB_KCAL
    vel = maxwell_boltzmann(rng, mass, 1.0)
    idx = np.arange(n, dtype=np.int64)
    return SystemDesc(pos=pos, vel=vel, mass=mass, boundary="PeriodicCuboid",
                      lower=(0.0, 0.0, 0.0), upper=(L, L, L), temperature=T,
                      ionic_strength=0.1,
                      lj=PairTerm("LennardJones", idx, np.ones(n), np.ones(n),
                                  cutoff=cutoff, margin=margin),
                      single_molecule=True, dt=dt, gamma=np.full(n, gamma), seed=seed)


def _synth(lib):
    """The library holding the seeded builders (include/mjolnir_b200_synthetic.h):
    `lib` when given (any ctypes library exporting the mjg_synth_* symbols),
    else libmjolnir_b200.so."""
    if lib is not None:
        return lib
    from . import _capi as A
    return A.lib()


def _f64(a):
    import ctypes as C
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _random_walk_chains(nchains, nbeads, bond, min_dist, radius, seed, synth=None):
    """Random-walk chains with `bond`-long steps from seed-drawn directions,
    rejecting any bead closer than `min_dist` to a bead other than the one it
    is bonded to, or outside the sphere of `radius` (native builder)."""
    out = np.empty((nchains * nbeads, 3))
    code = _synth(synth).mjg_synth_polymer_chains(nchains, nbeads, bond, min_dist, radius,
                                                  int(seed) & ((1 << 64) - 1), _f64(out))
    if code != 0:
        raise RuntimeError(f"mjg_synth_polymer_chains failed ({code}); lower the density")
    return out


def polymer_melt(nchains: int = 50, nbeads: int = 200, radius: float = 300.0,
                 charged_fraction: float = 0.2, temperature: float = 300.0,
                 ionic_strength: float = 0.1, dt: float = 0.01, gamma: float = 1.0,
                 margin: float = 0.5, seed: int = 2, mass: float = 1.0, synth=None) -> SystemDesc:
    """Coarse-grained polymer melt in unbounded space: harmonic bonds (k=100,
    r0=3.8), harmonic angles (k=10, 110 deg), cosine dihedrals (k=0.5, n=3,
    v0=0), ExcludedVolume (radius 2, eps 0.2, cutoff 2), DebyeHuckel on a
    random `charged_fraction` of beads with charges +-1 and zero net charge.
    `synth`: the library of the seeded builders (default libmjolnir_b200.so)."""
    rng = np.random.default_rng(seed)
    pos = _random_walk_chains(nchains, nbeads, 3.8, 4.0, radius, seed, synth)
    n = pos.shape[0]
    m = np.full(n, mass)
    vel = maxwell_boltzmann(rng, m, KB_KCAL * temperature)
    base = (np.arange(nchains, dtype=np.int64) * nbeads)[:, None]
    b = np.arange(nbeads - 1, dtype=np.int64)[None, :]
    bonds = np.stack([(base + b).ravel(), (base + b + 1).ravel()], axis=1)
    a = np.arange(nbeads - 2, dtype=np.int64)[None, :]
    angles = np.stack([(base + a).ravel(), (base + a + 1).ravel(), (base + a + 2).ravel()], axis=1)
    d = np.arange(nbeads - 3, dtype=np.int64)[None, :]
    dihd = np.stack([(base + d).ravel(), (base + d + 1).ravel(),
                     (base + d + 2).ravel(), (base + d + 3).ravel()], axis=1)
    nch = int(round(charged_fraction * n)) // 2 * 2
    charged = np.sort(rng.choice(n, size=nch, replace=False)).astype(np.int64)
    q = np.ones(nch)
    q[rng.permutation(nch)[: nch // 2]] = -1.0
    all_idx = np.arange(n, dtype=np.int64)
    return SystemDesc(
        pos=pos, vel=vel, mass=m, boundary="Unlimited", temperature=temperature,
        ionic_strength=ionic_strength,
        exv=PairTerm("ExcludedVolume", all_idx, np.full(n, 2.0), cutoff=2.0,
                     margin=margin, epsilon=0.2),
        dh=PairTerm("DebyeHuckel", charged, q, cutoff=5.5, margin=margin),
        ignore_molecule="Nothing", ignore_bond_within=3,
        bonds=(bonds, np.full(len(bonds), 100.0), np.full(len(bonds), 3.8)),
        angles=(angles, np.full(len(angles), 10.0), np.full(len(angles), math.radians(110.0))),
        dihedrals=(dihd, np.full(len(dihd), 0.5), np.full(len(dihd), 3, dtype=np.int32),
                   np.zeros(len(dihd))),
        dt=dt, gamma=np.full(n, gamma), seed=seed)


def bead_fluid(n: int = 1 << 20, density: float = 0.003, charged_fraction: float = 0.3,
               temperature: float = 300.0, ionic_strength: float = 0.15,
               dt: float = 0.3, gamma: float = 1.0, margin: float = 0.5,
               min_dist: float = 4.0, mass: float = 100.0, seed: int = 3, synth=None) -> SystemDesc:
    """Periodic EXV + Debye-Hueckel bead fluid: cubic box at number density
    `density`, uniform positions with overlaps below `min_dist` redrawn, charges
    +-1 on `charged_fraction` of the beads with zero net charge.  `synth`: the
    library of the seeded builders (default libmjolnir_b200.so)."""
    rng = np.random.default_rng(seed)
    L = (n / density) ** (1.0 / 3.0)
    pos = np.empty((n, 3))
    code = _synth(synth).mjg_synth_uniform_fluid(n, L, min_dist, int(seed) & ((1 << 64) - 1), _f64(pos))
    if code != 0:
        raise RuntimeError(f"mjg_synth_uniform_fluid failed ({code})")
    m = np.full(n, mass)
    vel = maxwell_boltzmann(rng, m, KB_KCAL * temperature)
    nch = int(round(charged_fraction * n)) // 2 * 2
    charged = np.sort(rng.choice(n, size=nch, replace=False)).astype(np.int64)
    q = np.ones(nch)
    q[rng.permutation(nch)[: nch // 2]] = -1.0
    all_idx = np.arange(n, dtype=np.int64)
    return SystemDesc(
        pos=pos, vel=vel, mass=m, boundary="PeriodicCuboid", lower=(0.0, 0.0, 0.0),
        upper=(L, L, L), temperature=temperature, ionic_strength=ionic_strength,
        exv=PairTerm("ExcludedVolume", all_idx, np.full(n, 2.0), cutoff=2.0,
                     margin=margin, epsilon=0.2),
        dh=PairTerm("DebyeHuckel", charged, q, cutoff=5.5, margin=margin),
        single_molecule=True, dt=dt, gamma=np.full(n, gamma), seed=seed)


def polymer_batch(nsys: int = 256, nmin: int = 500, nmax: int = 20000, seed: int = 4,
                  beads_per_chain: int = 200, dt: float = 0.01, gamma: float = 1.0,
                  margin: float = 0.5, synth=None):
    """Independent polymer melts built like :func:`polymer_melt`, sizes drawn
    log-uniform in [nmin, nmax] (chains of ~200 beads; the sphere radius keeps
    the 10,000-beads-in-300-A density), temperature U[280, 360] K and ionic
    strength U[0.05, 0.3] M per system.  `synth`: the library of the seeded
    builders (default libmjolnir_b200.so)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(nmin), np.log(nmax), nsys))
    temps = rng.uniform(280.0, 360.0, nsys)
    ions = rng.uniform(0.05, 0.3, nsys)
    out = []
    for k in range(nsys):
        nchains = max(1, int(round(sizes[k] / beads_per_chain)))
        nbeads = max(4, int(round(sizes[k] / nchains)))
        radius = 300.0 * (nchains * nbeads / 10000.0) ** (1.0 / 3.0)
        out.append(polymer_melt(nchains=nchains, nbeads=nbeads, radius=radius,
                                temperature=float(temps[k]), ionic_strength=float(ions[k]),
                                dt=dt, gamma=gamma, margin=margin, seed=seed * 100003 + k,
                                synth=synth))
    return out


def dimers(n: int = 20000, k: float = 0.5, r0: float = 3.8, temperature: float = 300.0,
           dt: float = 0.05, gamma: float = 1.0, integrator: str = "BAOAB", seed: int = 1) -> SystemDesc:
    """`n` independent harmonic dimers (mass 1, E = k (r - r0)^2, random
    orientations, 20 A apart on a line, no pair terms) for sampling tests:
    the bond length samples P(r) ~ r^2 exp(-k (r - r0)^2 / kB T).  For
    G-JFLangevin `gamma` is used as alpha (mass 1)."""
    rng = np.random.default_rng(seed)
    centers = np.stack([np.arange(n) * 20.0, np.zeros(n), np.zeros(n)], 1)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    pos = np.empty((2 * n, 3))
    pos[0::2] = centers - 0.5 * r0 * u
    pos[1::2] = centers + 0.5 * r0 * u
    m = np.ones(2 * n)
    idx = np.stack([np.arange(0, 2 * n, 2), np.arange(1, 2 * n, 2)], 1).astype(np.int64)
    return SystemDesc(pos=pos, vel=maxwell_boltzmann(rng, m, KB_KCAL * temperature), mass=m,
                      temperature=temperature, bonds=(idx, np.full(n, k), np.full(n, r0)),
                      integrator=integrator, dt=dt, gamma=np.full(2 * n, gamma), seed=seed)


def dimer_length_cdf(r: np.ndarray, k: float, r0: float, temperature: float) -> np.ndarray:
    """Cumulative Boltzmann distribution of a harmonic dimer's bond length at
    `r` (numerical integral of r^2 exp(-k (r - r0)^2 / kB T))."""
    beta = 1.0 / (KB_KCAL * temperature)
    w = 12.0 / np.sqrt(beta * k)
    grid = np.linspace(max(0.0, r0 - w), r0 + w, 400001)
    p = grid * grid * np.exp(-beta * k * (grid - r0) ** 2)
    c = np.concatenate([[0.0], np.cumsum(0.5 * (p[1:] + p[:-1]))])
    return np.interp(r, grid, c / c[-1])
