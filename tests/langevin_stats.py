"""Two-sample comparison of Langevin observables (kinetic temperature, per-term
potential energy) sampled along two runs of the same system with different
noise streams: the reference's mt19937 and this library's Philox.

Samples along a trajectory are correlated, so the means are compared with
block averages: the samples are cut into BLOCKS consecutive blocks, the
standard error of the mean is the spread of the block means over sqrt(BLOCKS),
and the two means must agree within Z_MAX combined standard errors.  For
"fast" observables, whose samples are further apart than their relaxation
time (the kinetic temperature, the bond and angle energies, the fluid's
energy), the widths (standard deviations) must also agree within WIDTH_TOL
relative and a two-sample Kolmogorov-Smirnov test must not reject at P_MIN.
Slow observables (a melt's dihedral, excluded-volume and electrostatic
energies, which follow the chains' conformations over the whole run) are
compared by their block means only.
"""
import numpy as np

BLOCKS = 10
Z_MAX = 5.0
WIDTH_TOL = 0.3
P_MIN = 1e-3


def block_mean(x):
    b = np.array_split(np.asarray(x, dtype=np.float64), BLOCKS)
    m = np.array([v.mean() for v in b])
    return float(m.mean()), float(m.std(ddof=1) / np.sqrt(BLOCKS))


def compare(a, b, fast=True):
    """Returns (ok, report) for samples a (this library) against b (the
    reference)."""
    from scipy import stats
    ma, sa = block_mean(a)
    mb, sb = block_mean(b)
    se = float(np.hypot(sa, sb))
    z = abs(ma - mb) / se if se > 0 else (0.0 if ma == mb else np.inf)
    wa, wb = float(np.std(a)), float(np.std(b))
    width = abs(wa / wb - 1.0) if wb > 0 else abs(wa)
    p = float(stats.ks_2samp(a, b).pvalue) if fast else None
    ok = z <= Z_MAX and (not fast or (width <= WIDTH_TOL and p >= P_MIN))
    return ok, {"mean": ma, "ref_mean": mb, "z": z, "width_rel": width, "ks_p": p}
