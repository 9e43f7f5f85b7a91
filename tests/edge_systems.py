"""Small systems at the edges of the cell-list and pair code: the smallest
periodic grid (3 cells per axis), particles exactly on cell and box
boundaries and outside the box, one- and two-particle systems, a term with no
participants, and clusters far apart in unbounded space (hashed-grid
aliasing).  Shared by the oracle-vs-reference and GPU-vs-oracle tests."""
import numpy as np

from mjolnir_b200 import systems as S


def _lj(pos, L, margin=0.5, seed=1):
    n = pos.shape[0]
    idx = np.arange(n, dtype=np.int64)
    rng = np.random.default_rng(seed)
    return S.SystemDesc(pos=pos, vel=rng.normal(size=(n, 3)), mass=np.ones(n), boundary="PeriodicCuboid",
                        lower=(0.0, 0.0, 0.0), upper=(L, L, L), temperature=1.0 / S.KB_KCAL,
                        lj=S.PairTerm("LennardJones", idx, np.ones(n), np.ones(n), cutoff=2.5, margin=margin),
                        single_molecule=True, dt=0.005, gamma=np.ones(n), seed=seed)


def _spread(n, L, dmin, seed):
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        p = rng.uniform(0, L, 3)
        d = np.array(out) - p if out else np.zeros((0, 3))
        d -= L * np.round(d / L)
        if not out or np.min(np.sum(d * d, axis=1)) >= dmin * dmin:
            out.append(p)
    return np.array(out)


def tiny_periodic():
    # cell width 2.5 (1 + 0.5) = 3.75 and L = 11.25: three cells per axis
    L = 11.25
    return _lj(_spread(40, L, 0.95, 3), L)


def on_boundaries():
    # particles on cell faces (multiples of the cell width), on the box's
    # lower faces, just below its upper faces, and outside it (wrapped in)
    L = 15.0
    w = L / 4
    pts = []
    for i in range(4):
        for j in range(4):
            pts.append([i * w, j * w, 0.0])
    pts += [[L - 1e-12, 1.0, 2.0], [-0.5, 7.0, 7.0], [L + 0.5, 3.0, 11.0], [7.5, -2.0, L + 1.0],
            [np.nextafter(w, 0.0), 5.0, 5.0], [np.nextafter(2 * w, 3 * w), 9.0, 9.0]]
    return _lj(np.array(pts, dtype=np.float64), L)


def exv_chain(n, spacing, radius_sep=None, seed=2):
    pos = np.zeros((n, 3))
    pos[:, 0] = np.arange(n) * spacing
    if radius_sep is not None:
        pos[n // 2:, :] += radius_sep
    idx = np.arange(n, dtype=np.int64)
    rng = np.random.default_rng(seed)
    return S.SystemDesc(pos=pos, vel=rng.normal(size=(n, 3)) * 0.1, mass=np.ones(n),
                        exv=S.PairTerm("ExcludedVolume", idx, np.full(n, 2.0), cutoff=2.0, margin=0.5,
                                       epsilon=0.2),
                        single_molecule=True, dt=0.01, gamma=np.ones(n), seed=seed)


def single():
    return exv_chain(1, 3.0)


def two():
    return exv_chain(2, 5.0)


def far_clusters():
    # two groups of 30 beads 5,000 A apart around (1e4, -1e4, 3e3): the
    # unbounded grid hashes both groups onto the same cells
    rng = np.random.default_rng(8)
    a = _spread(30, 25.0, 3.9, 8) + np.array([1e4, -1e4, 3e3])
    b = a + np.array([5000.0, 0.0, 0.0])
    pos = np.concatenate([a, b])
    n = pos.shape[0]
    idx = np.arange(n, dtype=np.int64)
    return S.SystemDesc(pos=pos, vel=rng.normal(size=(n, 3)) * 0.1, mass=np.ones(n),
                        exv=S.PairTerm("ExcludedVolume", idx, np.full(n, 2.0), cutoff=2.0, margin=0.5,
                                       epsilon=0.2),
                        single_molecule=True, dt=0.01, gamma=np.ones(n), seed=8)


def empty_dh():
    # a polymer whose DebyeHuckel term lists no charged bead
    d = S.polymer_melt(nchains=3, nbeads=20, radius=30.0, seed=12)
    d.dh = S.PairTerm("DebyeHuckel", np.zeros(0, dtype=np.int64), np.zeros(0), cutoff=5.5, margin=0.5)
    return d


CASES = {"tiny_periodic": tiny_periodic, "on_boundaries": on_boundaries, "single": single, "two": two,
         "far_clusters": far_clusters, "empty_dh": empty_dh}
