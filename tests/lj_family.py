"""Small periodic fluids for the Lennard-Jones family of the third global
term: LennardJones, WCA, LennardJonesAttractive (per-particle sigma and
epsilon, combined by the Lorentz-Berthelot rule) and UniformLennardJones
(one sigma and epsilon)."""
import numpy as np

from mjolnir_b200 import systems as S

KINDS = ("LennardJones", "WCA", "LennardJonesAttractive", "UniformLennardJones")


def fluid(kind, n=343, density=0.7, seed=5):
    d = S.lj_fluid(n=n, density=density, seed=seed, jitter=0.08)
    rng = np.random.default_rng(seed)
    idx = d.lj.idx
    if kind == "UniformLennardJones":
        sig, eps = np.full(n, 1.05), np.full(n, 0.8)
    else:
        sig = rng.choice([0.9, 1.0, 1.1], size=n)           # mixed sizes: sigma_ij = mean
        eps = rng.choice([0.5, 1.0, 1.0, 1.5], size=n)       # equal and unequal epsilons
    cutoff = {"WCA": 1.12246204831}.get(kind, 2.5)
    d.lj = S.PairTerm(kind, idx, sig, eps, cutoff=cutoff, margin=0.4)
    return d
