"""Small systems for the ExcludedVolume family of the first global term:
InversePower (n = 12 and n = 6) and HardCoreExcludedVolume, in a periodic
bead fluid and an unbounded polymer melt."""
import numpy as np

from mjolnir_b200 import systems as S

CASES = ("InversePower12", "InversePower6", "HardCoreExcludedVolume")


def system(case, periodic=True, seed=6):
    if periodic:
        d = S.bead_fluid(n=1500, density=0.004, seed=seed, dt=0.3)
    else:
        d = S.polymer_melt(nchains=4, nbeads=40, radius=40.0, seed=seed)
    idx = d.exv.idx
    n = len(idx)
    rng = np.random.default_rng(seed)
    radius = rng.choice([1.8, 2.0, 2.2], size=n)
    if case.startswith("InversePower"):
        power = int(case[len("InversePower"):])
        cutoff = 2.0 ** (12 // power)                       # InversePowerPotential default
        d.exv = S.PairTerm("InversePower", idx, radius, cutoff=cutoff, margin=0.4, epsilon=0.3,
                           exponent=power)
    else:
        shell = radius * 0.6                                  # soft shells 1.1-1.3 A
        core = rng.choice([0.5, 0.7], size=n)                 # hard cores well inside 4 A
        d.exv = S.PairTerm("HardCoreExcludedVolume", idx, shell, core, cutoff=2.0, margin=0.4,
                           epsilon=0.25)
    return d
