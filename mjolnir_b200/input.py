"""Reader (and writer) of the reference's TOML input for the per-step path.

``load(path)`` reads a Mjolnir input file the way input/read_input_file.hpp
does, for the subset of the schema that this library runs, and returns an
:class:`Input` whose ``desc`` is a :class:`~mjolnir_b200.systems.SystemDesc`
ready for :meth:`Engine.add_system`:

* ``[files]``: ``input.path`` (where included files are looked up;
  input/read_path.hpp:25-52), ``output.prefix``, ``output.path`` and
  ``output.format`` (``"xyz"``, ``"dcd"``, ``"trr"`` or an array of them;
  :mod:`mjolnir_b200.observers`);
* ``include = "f.toml"`` / ``["a.toml", ...]`` in any table, merged into it
  (input/utility.hpp:244-318), and ``file_name`` tables
  (input/read_table_from_file.hpp:38-91);
* ``[units]``: ``length = "angstrom"`` and ``energy = "kcal/mol"`` only (the
  constants of input/read_units.hpp:32-91 for those units are built in);
* ``[simulator]``: ``type = "MolecularDynamics"`` or ``"SimulatedAnnealing"``
  (``schedule = {type = "linear", begin, end}``, ``each_step``), ``boundary_type``,
  ``precision``, ``parallelism``, ``seed`` (or the deprecated
  ``integrator.seed``), ``delta_t``, ``total_step``, ``save_step``,
  ``integrator.type`` = ``"BAOABLangevin"`` or ``"UnderdampedLangevin"``
  (``gammas`` or the deprecated ``parameters``, input/read_integrator.hpp:55-187),
  ``"G-JFLangevin"`` (``alphas`` or ``parameters``, :242-300),
  ``"g-BAOABLangevin"`` (``gammas``, :189-239; without constraints, which the
  reader rejects) or ``"VelocityVerlet"``;
* ``[[systems]]`` (the first): ``attributes``, ``boundary_shape``,
  ``particles`` with ``mass|m``, ``position|pos``, ``velocity|vel``, ``name``,
  ``group`` (input/read_system.hpp:93-290), or ``file_name = "x.msg"``, a
  checkpoint in the reference's MsgPack layout (:mod:`mjolnir_b200.checkpoint`);
* ``[[forcefields]]`` (the first): ``[[forcefields.local]]`` BondLength /
  BondAngle with Harmonic (``k``, ``v0``) and DihedralAngle with Cosine
  (``k``, ``n``, ``v0``), ``indices`` plus an optional ``offset``
  (input/read_local_potential.hpp:473-522); ``[[forcefields.global]]`` Pair
  with ExcludedVolume (``epsilon``, ``radius``), InversePower (``epsilon``,
  ``n``, ``radius``; cutoff default 2^(12/n)), HardCoreExcludedVolume
  (``epsilon``, ``soft_shell_thickness``, ``core_radius``), DebyeHuckel (``charge``),
  LennardJones, WCA or LennardJonesAttractive (``sigma|σ``, ``epsilon|ε``) or
  UniformLennardJones (global ``sigma``, ``epsilon``; ``parameters`` optional),
  ``cutoff`` (defaults 2.0 / 5.5 / 2.5; WCA's is fixed at 2^(1/6)),
  ``spatial_partition = {type = "CellList"|"VerletList", margin}``,
  ``ignore.molecule`` and ``ignore.particles_within``
  (input/read_global_potential.hpp:32-300,360-470,660-705).

Parameters may name a value of the table's ``env`` instead of giving it
(input/utility.hpp:26-58).  Anything else in those tables (other
potentials, ``ignore.group``, external or constraint force fields, other
simulators or integrators, other units) raises :class:`InputError` naming
the key: the per-step path does not run it, and silently dropping a term
would change the physics.

When the particles carry no velocities the reference draws them from a
Maxwell-Boltzmann distribution with its mt19937 stream (core/System.hpp:58-95);
here they are drawn from numpy's PCG64 seeded with ``simulator.seed`` — the
same distribution, not the same numbers.
"""
from __future__ import annotations

import dataclasses
import os
import tomllib
from typing import Optional

import numpy as np

from .systems import KB_KCAL, PairTerm, SystemDesc

DEFAULT_CUTOFF = {"ExcludedVolume": 2.0, "HardCoreExcludedVolume": 2.0, "InversePower": None,
                  "DebyeHuckel": 5.5, "LennardJones": 2.5,
                  "WCA": 1.12246204831, "LennardJonesAttractive": 2.5, "UniformLennardJones": 2.5}
LJ_FAMILY = ("LennardJones", "WCA", "LennardJonesAttractive", "UniformLennardJones")
LOCAL_FORMS = {("BondLength", "Harmonic"): 2, ("BondAngle", "Harmonic"): 3,
               ("DihedralAngle", "Cosine"): 4}


class InputError(ValueError):
    """The input uses something outside the per-step path, or is malformed."""


@dataclasses.dataclass
class Input:
    desc: SystemDesc
    simulator: str                  # "MolecularDynamics" | "SimulatedAnnealing"
    precision: str                  # "double" | "float"
    parallelism: str
    total_step: int
    save_step: int
    seed: int
    output_prefix: str
    output_path: str                # ends with "/" (input/read_path.hpp:56-75)
    output_formats: list            # "xyz" | "dcd" | "trr", in input order
    input_path: str
    schedule: Optional[tuple] = None   # SimulatedAnnealing: (first, last, each_step)
    checkpoint_step: int = 0           # checkpoint interval (default: save_step)
    names: Optional[list] = None       # particle names (default "X")
    groups: Optional[list] = None      # particle groups (default "NONE")
    attributes: Optional[dict] = None  # [[systems]] attributes as given (temperature, ionic_strength, ...)

    @property
    def file_prefix(self) -> str:
        """output path + prefix, the stem of every output file
        (input/read_observer.hpp:68-74)."""
        return self.output_path + self.output_prefix


# ------------------------------------------------------------------ helpers
def _parse(path: str) -> dict:
    try:
        with open(path, "rb") as f:
            return tomllib.load(f)
    except FileNotFoundError:
        raise InputError(f"file not found: {path}") from None
    except tomllib.TOMLDecodeError as e:
        raise InputError(f"{path}: {e}") from None


def _resolve(input_path: str, name: str, base_dir: str) -> str:
    """The reference opens ``input_path + name`` relative to the working
    directory; a path that does not exist there is also tried relative to
    the directory of the main input file."""
    p = input_path + name
    if os.path.isabs(p) or os.path.exists(p):
        return p
    alt = os.path.join(base_dir, p)
    return alt if os.path.exists(alt) else p


def _merge(table: dict, other: dict, where: str):
    for k, v in other.items():
        if k in table:
            if isinstance(table[k], dict) and isinstance(v, dict):
                _merge(table[k], v, f"{where}.{k}")
            else:
                raise InputError(f'value "{k}" duplicates in {where}')
        else:
            table[k] = v


def _expand_include(v, input_path: str, base_dir: str, where: str = "root"):
    if isinstance(v, dict):
        for k, x in list(v.items()):
            if k != "include":
                _expand_include(x, input_path, base_dir, f"{where}.{k}")
        if "include" in v:
            inc = v.pop("include")
            for name in (inc if isinstance(inc, list) else [inc]):
                if not isinstance(name, str):
                    raise InputError(f"{where}.include must be a string or an array of strings")
                _merge(v, _parse(_resolve(input_path, name, base_dir)), where)
    elif isinstance(v, list):
        for k, x in enumerate(v):
            _expand_include(x, input_path, base_dir, f"{where}[{k}]")


def _from_file(table: dict, name: str, input_path: str, base_dir: str) -> dict:
    if not isinstance(table, dict):
        raise InputError(f"[{name}] must be a table")
    if "file_name" not in table:
        return table
    other = _parse(_resolve(input_path, table["file_name"], base_dir))
    if name not in other:
        raise InputError(f"table [{name}] not found in {table['file_name']}")
    t = other[name]
    if isinstance(t, list):
        if len(t) != 1:
            raise InputError(f"{table['file_name']} should define exactly one [[{name}]]")
        t = t[0]
    return t


def _check_keys(table: dict, allowed, where: str):
    extra = set(table) - set(allowed)
    if extra:
        raise InputError(f"{where}: unsupported key(s) {sorted(extra)}")


def _param(item: dict, env: Optional[dict], *names, default=None, where=""):
    """find_parameter: the first of `names` present; a string value names an
    entry of `env`."""
    for nm in names:
        if nm in item:
            v = item[nm]
            if isinstance(v, str):
                if env is None:
                    raise InputError(f'{where}: named variable "{v}" used but no env is defined')
                if v not in env:
                    raise InputError(f'{where}: named variable "{v}" does not exist in env')
                return env[v]
            return v
    if default is not None:
        return default
    raise InputError(f"{where}: value {' or '.join(names)} does not exist")


def _index(item, env, where):
    return int(_param(item, env, "index", where=where)) + int(_param(item, env, "offset", default=0, where=where))


def _no_overlap(idx, where):
    if len(set(idx)) != len(idx):
        raise InputError(f"{where}: an index appears twice")


# ------------------------------------------------------------------ sections
def _units(root):
    u = root.get("units", {})
    _check_keys(u, {"length", "energy"}, "[units]")
    if u.get("length", "angstrom") not in ("angstrom", "Å", "angstorm"):
        raise InputError('[units] length: only "angstrom" is supported')
    if u.get("energy", "kcal/mol") != "kcal/mol":
        raise InputError('[units] energy: only "kcal/mol" is supported')


def _simulator(sim):
    typ = sim.get("type")
    keys = {"type", "boundary_type", "precision", "parallelism", "seed", "total_step",
            "save_step", "checkpoint_step", "delta_t", "integrator", "forcefields", "env"}
    if typ == "SimulatedAnnealing":                 # input/read_simulator.hpp:84-160
        keys |= {"schedule", "each_step"}
    elif typ != "MolecularDynamics":
        raise InputError(f'[simulator] type "{typ}": only "MolecularDynamics" and '
                         '"SimulatedAnnealing" are supported')
    _check_keys(sim, keys, "[simulator]")
    bt = sim.get("boundary_type")
    if bt not in ("Unlimited", "Periodic", "PeriodicCuboid"):
        raise InputError(f'[simulator] boundary_type "{bt}" is not one of Unlimited, PeriodicCuboid')
    prec = sim.get("precision")
    if prec not in ("double", "float"):
        raise InputError(f'[simulator] precision "{prec}" is not "double" or "float"')
    par = sim.get("parallelism", "sequencial")
    if par not in ("sequencial", "openmp", "OpenMP"):
        raise InputError(f'[simulator] parallelism "{par}" is not "sequencial" or "openmp"')
    integ = sim.get("integrator")
    if not isinstance(integ, dict) or "type" not in integ:
        raise InputError("[simulator] integrator.type is required")
    if "seed" in integ:
        seed = int(integ["seed"])                   # deprecated location
    else:
        seed = int(sim.get("seed", 0))
    for k in ("delta_t", "total_step", "save_step"):
        if k not in sim:
            raise InputError(f"[simulator] {k} is required")
    return bt, prec, par, integ, seed


def _integrator(integ, n):
    kind = integ["type"]
    if kind == "VelocityVerlet":
        _check_keys(integ, {"type", "seed", "remove"}, "[simulator.integrator]")
        return "VelocityVerlet", np.zeros(n)
    if kind not in _LANGEVIN:
        raise InputError(f'integrator type "{kind}": only "BAOABLangevin", "UnderdampedLangevin", '
                         '"G-JFLangevin", "g-BAOABLangevin" and "VelocityVerlet" are supported')
    name, plural, single, alt = _LANGEVIN[kind]
    _check_keys(integ, {"type", "seed", "remove", "env", "parameters", plural}, "[simulator.integrator]")
    if "parameters" in integ and plural in integ:
        raise InputError(f'duplicated keys: both "parameters" and "{plural}" are provided')
    items = integ.get(plural, integ.get("parameters"))
    if items is None:
        raise InputError(f"{kind} needs {plural}")
    env = integ.get("env")
    idx = [_index(it, env, f"integrator.{plural}") for it in items]
    _no_overlap(idx, f"integrator.{plural}")
    gamma = np.zeros(max(n, max(idx, default=-1) + 1))
    for i, it in zip(idx, items):
        gamma[i] = float(_param(it, env, *[k for k in (single, alt) if k], where=f"integrator.{plural}"))
    if gamma.shape[0] != n:
        raise InputError(f"integrator.{plural} index {gamma.shape[0] - 1} is out of range")
    return name, gamma


# integrator type -> (SystemDesc.integrator, list key, parameter key, its
# alternative spelling); input/read_integrator.hpp:55-187, 242-300
_LANGEVIN = {"BAOABLangevin": ("BAOAB", "gammas", "gamma", "γ"),
             "UnderdampedLangevin": ("UnderdampedLangevin", "gammas", "gamma", "γ"),
             "G-JFLangevin": ("G-JFLangevin", "alphas", "alpha", None),
             "g-BAOABLangevin": ("g-BAOABLangevin", "gammas", "gamma", "γ")}


def _system(sysd, boundary):
    _check_keys(sysd, {"boundary_shape", "attributes", "dynamic_variables", "particles"}, "[[systems]]")
    if sysd.get("dynamic_variables"):
        raise InputError("[[systems]] dynamic_variables are not supported")
    parts = sysd.get("particles")
    if not parts:
        raise InputError("[[systems]] particles are required")
    n = len(parts)
    pos = np.empty((n, 3))
    mass = np.empty(n)
    has_vel = "velocity" in parts[0] or "vel" in parts[0]
    vel = np.zeros((n, 3))
    names, groups = [], []
    for i, p in enumerate(parts):
        _check_keys(p, {"mass", "m", "position", "pos", "velocity", "vel", "name", "group"}, f"particle {i}")
        mass[i] = float(p["m"] if "m" in p else p["mass"])
        pos[i] = p["pos"] if "pos" in p else p["position"]
        pv = "velocity" in p or "vel" in p
        if pv != has_vel:
            raise InputError("read_system: give velocity for all particles or for none")
        if pv:
            vel[i] = p["vel"] if "vel" in p else p["velocity"]
        names.append(str(p.get("name", "X")))          # read_system.hpp:276-277
        groups.append(str(p.get("group", "NONE")))
    attrs = sysd.get("attributes", {})
    shape = sysd.get("boundary_shape", {})
    lower = upper = (0.0, 0.0, 0.0)
    if boundary == "PeriodicCuboid":
        _check_keys(shape, {"lower", "upper"}, "[[systems]] boundary_shape")
        lower = tuple(float(x) for x in shape["lower"])
        upper = tuple(float(x) for x in shape["upper"])
        if not all(u > lo for u, lo in zip(upper, lower)):
            raise InputError("boundary_shape: upper must exceed lower on every axis")
    elif shape:
        raise InputError("boundary_shape must be empty for an Unlimited boundary")
    return pos, vel, mass, has_vel, attrs, lower, upper, names, groups


def _ignore(g, where):
    ign = g.get("ignore", {})
    _check_keys(ign, {"molecule", "group", "particles_within"}, f"{where}.ignore")
    grp = ign.get("group", {})
    if grp and (grp.get("intra") or grp.get("inter")):
        raise InputError(f"{where}: ignore.group is not supported")
    mol = ign.get("molecule", "Nothing")
    if mol not in ("Nothing", "Self", "Intra", "Others", "Inter"):
        raise InputError(f'{where}: ignore.molecule "{mol}" is not Nothing, Self or Others')
    within = {str(k): int(v) for k, v in ign.get("particles_within", {}).items()}
    return mol, within


def _global(g, n, where):
    inter = g.get("interaction")
    pot = g.get("potential")
    if inter != "Pair" or pot not in DEFAULT_CUTOFF:
        raise InputError(f'{where}: "{inter}" / "{pot}" is not run here (Pair with ExcludedVolume, '
                         "DebyeHuckel, LennardJones, WCA, LennardJonesAttractive or UniformLennardJones)")
    allowed = {"interaction", "potential", "ignore", "spatial_partition", "parameters", "env", "cutoff"}
    if pot in ("ExcludedVolume", "UniformLennardJones", "InversePower", "HardCoreExcludedVolume"):
        allowed |= {"epsilon"}
    if pot == "InversePower":
        allowed |= {"n"}
    if pot == "UniformLennardJones":
        allowed |= {"sigma"}
    if "table" in g:
        raise InputError(f"{where}: parameter tables are not supported")
    _check_keys(g, allowed, where)
    sp = g.get("spatial_partition")
    if not isinstance(sp, dict) or sp.get("type") not in ("CellList", "VerletList"):
        raise InputError(f'{where}: spatial_partition.type must be "CellList" or "VerletList"')
    margin = float(sp["margin"])
    env = g.get("env")
    if pot == "UniformLennardJones" and "parameters" not in g:
        items = [{"index": i} for i in range(n)]   # every particle (EmptyCombinationRule)
    else:
        items = g.get("parameters", [])
    idx = np.array([_index(it, env, where) for it in items], dtype=np.int64)
    _no_overlap(idx.tolist(), where)
    if idx.size and (idx.min() < 0 or idx.max() >= n):
        raise InputError(f"{where}: participant index out of range")
    # WCA's cutoff is fixed (input/read_global_potential.hpp warns and ignores it);
    # InversePower's default is 2^(12 / n) with an integer quotient
    # (InversePowerPotential.hpp:27-30)
    if pot == "InversePower":
        if "n" not in g or "epsilon" not in g:
            raise InputError(f"{where}: InversePower needs epsilon and n")
        power = int(g["n"])
        if power <= 0:
            raise InputError(f"{where}: InversePower n must be positive")
        cutoff = float(g.get("cutoff", 2.0 ** (12 // power)))
    else:
        cutoff = DEFAULT_CUTOFF[pot] if pot == "WCA" else float(g.get("cutoff", DEFAULT_CUTOFF[pot]))
    mol, within = _ignore(g, where)
    if pot in ("ExcludedVolume", "InversePower"):
        if "epsilon" not in g:
            raise InputError(f"{where}: {pot} needs epsilon")
        p0 = np.array([float(_param(it, env, "radius", where=where)) for it in items])
        term = PairTerm(pot, idx, p0, cutoff=cutoff, margin=margin, epsilon=float(g["epsilon"]),
                        exponent=power if pot == "InversePower" else 12)
    elif pot == "HardCoreExcludedVolume":
        if "epsilon" not in g:
            raise InputError(f"{where}: HardCoreExcludedVolume needs epsilon")
        p0 = np.array([float(_param(it, env, "soft_shell_thickness", where=where)) for it in items])
        p1 = np.array([float(_param(it, env, "core_radius", where=where)) for it in items])
        term = PairTerm(pot, idx, p0, p1, cutoff=cutoff, margin=margin, epsilon=float(g["epsilon"]))
    elif pot == "DebyeHuckel":
        p0 = np.array([float(_param(it, env, "charge", where=where)) for it in items])
        term = PairTerm(pot, idx, p0, cutoff=cutoff, margin=margin)
    elif pot == "UniformLennardJones":
        for k in ("sigma", "epsilon"):
            if k not in g:
                raise InputError(f"{where}: UniformLennardJones needs {k}")
        p0 = np.full(len(idx), float(g["sigma"]))
        p1 = np.full(len(idx), float(g["epsilon"]))
        term = PairTerm(pot, idx, p0, p1, cutoff=cutoff, margin=margin)
    else:
        p0 = np.array([float(_param(it, env, "sigma", "σ", where=where)) for it in items])
        p1 = np.array([float(_param(it, env, "epsilon", "ε", where=where)) for it in items])
        term = PairTerm(pot, idx, p0, p1, cutoff=cutoff, margin=margin)
    term.ignore_molecule = mol
    term.ignore_within = within
    return term


def _local(loc, n, where):
    inter, pot = loc.get("interaction"), loc.get("potential")
    arity = LOCAL_FORMS.get((inter, pot))
    if arity is None:
        raise InputError(f'{where}: "{inter}" with "{pot}" is not run here '
                         "(BondLength/BondAngle Harmonic, DihedralAngle Cosine)")
    _check_keys(loc, {"interaction", "potential", "topology", "parameters", "env"}, where)
    if "topology" not in loc:
        raise InputError(f"{where}: topology is required")
    env = loc.get("env")
    items = loc.get("parameters", [])
    allowed = {"indices", "k", "v0", "offset"} | ({"n"} if pot == "Cosine" else set())
    idx = np.empty((len(items), arity), dtype=np.int64)
    k = np.empty(len(items))
    v0 = np.empty(len(items))
    nn = np.empty(len(items), dtype=np.int32)
    for t, it in enumerate(items):
        _check_keys(it, allowed, where)
        ind = [int(x) for x in _param(it, env, "indices", where=where)]
        if len(ind) != arity:
            raise InputError(f"{where}: indices must have {arity} entries")
        off = _param(it, env, "offset", default=0, where=where)
        if isinstance(off, list):
            if len(off) != arity:
                raise InputError(f"{where}: invalid size of offset array")
            ind = [a + int(b) for a, b in zip(ind, off)]
        else:
            ind = [a + int(off) for a in ind]
        if min(ind) < 0 or max(ind) >= n:
            raise InputError(f"{where}: index out of range")
        idx[t] = ind
        k[t] = float(_param(it, env, "k", where=where))
        v0[t] = float(_param(it, env, "v0", where=where))
        if pot == "Cosine":
            nn[t] = int(_param(it, env, "n", where=where))
    return inter, str(loc["topology"]), idx, k, v0, nn


def _forcefield(ff, n, input_path, base_dir):
    _check_keys(ff, {"local", "global", "external", "constraint", "name"}, "[[forcefields]]")
    if ff.get("external") or ff.get("constraint"):
        raise InputError("[[forcefields]] external and constraint force fields are not run here")
    pairs = {}
    for i, g in enumerate(ff.get("global", [])):
        g = _from_file(g, "global", input_path, base_dir)
        t = _global(g, n, f"forcefields.global[{i}]")
        key = {"ExcludedVolume": "exv", "InversePower": "exv", "HardCoreExcludedVolume": "exv",
               "DebyeHuckel": "dh"}.get(t.kind, "lj")
        if key in pairs:
            family = {"exv": "ExcludedVolume-family", "dh": "DebyeHuckel", "lj": "Lennard-Jones-family"}[key]
            raise InputError(f"forcefields.global[{i}]: a second {family} term is not supported")
        pairs[key] = t
    locs = {}
    for i, loc in enumerate(ff.get("local", [])):
        loc = _from_file(loc, "local", input_path, base_dir)
        inter, topo, idx, k, v0, nn = _local(loc, n, f"forcefields.local[{i}]")
        if inter in locs:
            prev = locs[inter]
            if prev[0] != topo:
                raise InputError(f"forcefields.local[{i}]: {inter} terms with different topology "
                                 "kinds are not supported")
            locs[inter] = (topo, np.concatenate([prev[1], idx]), np.concatenate([prev[2], k]),
                           np.concatenate([prev[3], v0]), np.concatenate([prev[4], nn]))
        else:
            locs[inter] = (topo, idx, k, v0, nn)
    return pairs, locs


# ------------------------------------------------------------------ entry
def load(path: str) -> Input:
    """Reads a Mjolnir input file (see the module docstring for the subset)."""
    base_dir = os.path.dirname(os.path.abspath(path))
    root = _parse(path)
    _check_keys(root, {"files", "units", "simulator", "systems", "forcefields"}, "input")
    files = root.get("files", {})
    inp = files.get("input", {})
    input_path = inp.get("path", "./") if isinstance(inp, dict) else "./"
    if not input_path.endswith("/"):
        input_path += "/"
    out = files.get("output", {})
    out_path = str(out.get("path", "./"))
    if not out_path.endswith("/"):
        out_path += "/"
    fmt = out.get("format", "xyz")                 # read_observer.hpp:17-96: a string or an array
    formats = [fmt] if isinstance(fmt, str) else list(fmt)
    for f in formats:
        if f not in ("xyz", "dcd", "trr"):
            raise InputError(f'files.output.format "{f}": one of "xyz", "dcd" and "trr" is expected')
    _expand_include(root, input_path, base_dir)
    _units(root)
    sim = _from_file(root.get("simulator", {}), "simulator", input_path, base_dir)
    boundary, prec, par, integ, seed = _simulator(sim)
    boundary = "PeriodicCuboid" if boundary in ("Periodic", "PeriodicCuboid") else "Unlimited"
    systems = root.get("systems")
    if not systems:
        raise InputError("[[systems]] is required")
    first = systems[0]
    if isinstance(first, dict) and str(first.get("file_name", "")).endswith(".msg"):
        # a checkpoint (input/read_system.hpp:105-131): state, box and
        # attributes from the MsgPack file
        from .checkpoint import CheckpointError, read_system
        try:
            ck = read_system(_resolve(input_path, first["file_name"], base_dir))
        except CheckpointError as e:
            raise InputError(str(e)) from None
        if ck["periodic"] != (boundary == "PeriodicCuboid"):
            raise InputError("the checkpoint's boundary does not match [simulator] boundary_type")
        pos, vel, mass, has_vel = ck["pos"], ck["vel"], ck["mass"], True
        attrs, lower, upper = ck["attributes"], ck["lower"], ck["upper"]
        names, groups = ck["names"], ck["groups"]
    else:
        sysd = _from_file(first, "systems", input_path, base_dir)
        pos, vel, mass, has_vel, attrs, lower, upper, names, groups = _system(sysd, boundary)
    n = pos.shape[0]
    temperature = float(attrs.get("temperature", 300.0))
    ionic = float(attrs.get("ionic_strength", 0.1))
    ffs = root.get("forcefields")
    if not ffs:
        raise InputError("[[forcefields]] is required")
    pairs, locs = _forcefield(_from_file(ffs[0], "forcefields", input_path, base_dir), n,
                              input_path, base_dir)
    if "dh" in pairs and "ionic_strength" not in attrs:
        raise InputError("DebyeHuckel needs systems.attributes.ionic_strength")
    if pairs and not has_vel and "temperature" not in attrs:
        raise InputError("generating velocities needs systems.attributes.temperature")
    integrator, gamma = _integrator(integ, n)
    schedule = None
    if sim["type"] == "SimulatedAnnealing":
        sch = sim.get("schedule")
        if not isinstance(sch, dict) or "each_step" not in sim:
            raise InputError("SimulatedAnnealing needs [simulator] schedule and each_step")
        _check_keys(sch, {"type", "begin", "end", "each_step"}, "[simulator.schedule]")
        if sch.get("type") != "linear":
            raise InputError('schedule.type: only "linear" is supported')
        if integrator == "VelocityVerlet":
            raise InputError("SimulatedAnnealing needs a Langevin integrator")
        schedule = (float(sch["begin"]), float(sch["end"]), int(sim["each_step"]))
        temperature = schedule[0]                   # current(0), set before initialisation
    if boundary == "PeriodicCuboid":              # System::initialize wraps positions
        lo, up = np.array(lower), np.array(upper)
        w = up - lo
        pos = np.where(pos < lo, pos + w, np.where(pos >= up, pos - w, pos))
    if not has_vel:
        rng = np.random.default_rng(seed)
        vel = rng.standard_normal((n, 3)) * np.sqrt(KB_KCAL * temperature / mass)[:, None]
    desc = SystemDesc(pos=pos, vel=vel, mass=mass, boundary=boundary, lower=lower, upper=upper,
                      temperature=temperature, ionic_strength=ionic,
                      exv=pairs.get("exv"), dh=pairs.get("dh"), lj=pairs.get("lj"),
                      integrator=integrator, dt=float(sim["delta_t"]), gamma=gamma, seed=seed)
    # one rule shared by every pair term is kept system-wide as well
    rules = {(t.ignore_molecule, tuple(sorted(t.ignore_within.items()))) for t in pairs.values()}
    if len(rules) == 1:
        mol, within = rules.pop()
        w = dict(within)
        if set(w) <= {"bond"}:
            desc.ignore_molecule = mol
            desc.ignore_bond_within = int(w.get("bond", 0))
    if "BondLength" in locs:
        topo, idx, k, v0, _ = locs["BondLength"]
        desc.bonds, desc.bond_topology = (idx, k, v0), topo
    if "BondAngle" in locs:
        topo, idx, k, v0, _ = locs["BondAngle"]
        desc.angles, desc.angle_topology = (idx, k, v0), topo
    if "DihedralAngle" in locs:
        topo, idx, k, v0, nn = locs["DihedralAngle"]
        desc.dihedrals, desc.dihedral_topology = (idx, k, nn, v0), topo
    return Input(desc=desc, simulator=sim["type"], schedule=schedule, precision=prec, parallelism=par,
                 total_step=int(sim["total_step"]), save_step=int(sim["save_step"]), seed=seed,
                 checkpoint_step=int(sim.get("checkpoint_step", sim["save_step"])),
                 output_prefix=str(out.get("prefix", "mjolnir")), output_path=out_path,
                 output_formats=formats, input_path=input_path, names=names, groups=groups,
                 attributes={str(k): float(v) for k, v in attrs.items()})


# ------------------------------------------------------------------ writer
def _fmt(x) -> str:
    if isinstance(x, (bool, np.bool_)):
        return "true" if x else "false"
    if isinstance(x, (int, np.integer)):
        return str(int(x))
    if isinstance(x, (float, np.floating)):
        r = repr(float(x))
        if r in ("inf", "-inf", "nan"):
            raise ValueError("TOML cannot hold a non-finite value here")
        return r
    if isinstance(x, str):
        return '"' + x.replace("\\", "\\\\").replace('"', '\\"') + '"'
    if isinstance(x, (list, tuple, np.ndarray)):
        return "[" + ", ".join(_fmt(v) for v in x) + "]"
    raise TypeError(type(x))


def dumps(desc: SystemDesc, total_step: int = 1000, save_step: int = 100, prefix: str = "mjolnir",
          precision: str = "double") -> str:
    """Writes `desc` as one self-contained Mjolnir input file."""
    L = []
    a = L.append
    a("[files]")
    a(f"output.prefix = {_fmt(prefix)}")
    a('output.path = "./"')
    a('output.format = "xyz"')
    a("")
    a("[units]")
    a('length = "angstrom"')
    a('energy = "kcal/mol"')
    a("")
    a("[simulator]")
    a('type = "MolecularDynamics"')
    a(f"boundary_type = {_fmt(desc.boundary)}")
    a(f"precision = {_fmt(precision)}")
    a(f"seed = {int(desc.seed)}")
    a(f"delta_t = {_fmt(float(desc.dt))}")
    a(f"total_step = {int(total_step)}")
    a(f"save_step = {int(save_step)}")
    if desc.integrator == "VelocityVerlet":
        a('integrator.type = "VelocityVerlet"')
    else:
        kind = {v[0]: k for k, v in _LANGEVIN.items()}[desc.integrator]
        _, plural, single, _ = _LANGEVIN[kind]
        a(f'integrator.type = "{kind}"')
        g = desc.gamma if desc.gamma is not None else np.zeros(desc.n)
        a(f"integrator.{plural} = [")
        for i, x in enumerate(g):
            a(f"  {{index = {i}, {single} = {_fmt(float(x))}}},")
        a("]")
    a("")
    a("[[systems]]")
    a(f"attributes.temperature = {_fmt(float(desc.temperature))}")
    a(f"attributes.ionic_strength = {_fmt(float(desc.ionic_strength))}")
    if desc.periodic:
        a(f"boundary_shape.lower = {_fmt([float(x) for x in desc.lower])}")
        a(f"boundary_shape.upper = {_fmt([float(x) for x in desc.upper])}")
    a("particles = [")
    for i in range(desc.n):
        a(f"  {{mass = {_fmt(float(desc.mass[i]))}, position = {_fmt(desc.pos[i].tolist())}, "
          f"velocity = {_fmt(desc.vel[i].tolist())}}},")
    a("]")
    a("")
    a("[[forcefields]]")
    locals_ = [("BondLength", "Harmonic", desc.bond_topology, desc.bonds),
               ("BondAngle", "Harmonic", desc.angle_topology, desc.angles),
               ("DihedralAngle", "Cosine", desc.dihedral_topology, desc.dihedrals)]
    for inter, pot, topo, data in locals_:
        if data is None:
            continue
        a("[[forcefields.local]]")
        a(f"interaction = {_fmt(inter)}")
        a(f"potential = {_fmt(pot)}")
        a(f"topology = {_fmt(topo)}")
        a("parameters = [")
        if pot == "Cosine":
            idx, k, nn, v0 = data
            for t in range(len(k)):
                a(f"  {{indices = {_fmt(idx[t].tolist())}, k = {_fmt(float(k[t]))}, "
                  f"n = {int(nn[t])}, v0 = {_fmt(float(v0[t]))}}},")
        else:
            idx, k, v0 = data
            for t in range(len(k)):
                a(f"  {{indices = {_fmt(idx[t].tolist())}, k = {_fmt(float(k[t]))}, v0 = {_fmt(float(v0[t]))}}},")
        a("]")
    if desc.single_molecule and desc.n > 1:
        # the chain that makes a fluid one molecule is not an interaction; it
        # changes nothing when no rule looks at molecules or bonds
        rules = [(t.ignore_molecule if t.ignore_molecule is not None else desc.ignore_molecule,
                  (t.ignore_within or {}).get("bond", desc.ignore_bond_within if t.ignore_within is None else 0))
                 for t in desc.pair_terms()]
        if any(m != "Nothing" or w > 0 for m, w in rules):
            raise ValueError("a single-molecule system whose ignore rules use molecules or bonds "
                             "has no TOML form")
    for t in desc.pair_terms():
        a("[[forcefields.global]]")
        a('interaction = "Pair"')
        a(f"potential = {_fmt(t.kind)}")
        if t.kind != "WCA":
            a(f"cutoff = {_fmt(float(t.cutoff))}")
        if t.kind in ("ExcludedVolume", "InversePower", "HardCoreExcludedVolume"):
            a(f"epsilon = {_fmt(float(t.epsilon))}")
        if t.kind == "InversePower":
            a(f"n = {int(t.exponent)}")
        if t.kind == "UniformLennardJones":
            a(f"sigma = {_fmt(float(t.param0[0]))}")
            a(f"epsilon = {_fmt(float(t.param1[0]))}")
        a(f'spatial_partition = {{type = "CellList", margin = {_fmt(float(t.margin))}}}')
        mol = t.ignore_molecule if t.ignore_molecule is not None else desc.ignore_molecule
        within = t.ignore_within if t.ignore_within is not None else (
            {"bond": desc.ignore_bond_within} if desc.ignore_bond_within > 0 else {})
        a(f"ignore.molecule = {_fmt(mol)}")
        a("ignore.particles_within = {" + ", ".join(f"{k} = {int(v)}" for k, v in within.items()) + "}")
        a("parameters = [")
        name = {"ExcludedVolume": "radius", "InversePower": "radius", "DebyeHuckel": "charge",
                "HardCoreExcludedVolume": "soft_shell_thickness"}.get(t.kind, "sigma")
        for q in range(len(t.idx)):
            if t.kind == "UniformLennardJones":
                a(f"  {{index = {int(t.idx[q])}}},")
                continue
            if t.kind == "HardCoreExcludedVolume":
                a(f"  {{index = {int(t.idx[q])}, soft_shell_thickness = {_fmt(float(t.param0[q]))}, "
                  f"core_radius = {_fmt(float(t.param1[q]))}}},")
                continue
            extra = f", epsilon = {_fmt(float(t.param1[q]))}" if t.kind in LJ_FAMILY else ""
            a(f"  {{index = {int(t.idx[q])}, {name} = {_fmt(float(t.param0[q]))}{extra}}},")
        a("]")
    return "\n".join(L) + "\n"


def dump(desc: SystemDesc, path: str, **kw):
    with open(path, "w") as f:
        f.write(dumps(desc, **kw))

