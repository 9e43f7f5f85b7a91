"""CPU checkers for the Mjolnir hot path.  TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` use this package; the product path
(``mjolnir_b200``) never imports it.

* :class:`Oracle`    -- ctypes front end of ``liboracle.so``, the plain-C
  restatement of the reference algorithms (``oracle.c``).
* :class:`Reference` -- ctypes front end of ``_ref/libmjolnir_ref.so``, the
  reference's own code compiled from its unmodified headers
  (``ref_driver.cpp``); present only where the reference tree was available
  at build time.

Both take a duck-typed system description with the attributes of
``mjolnir_b200.systems.SystemDesc``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmjolnir_ref.so")

TERM_BOND, TERM_ANGLE, TERM_DIHEDRAL, TERM_EXV, TERM_DH, TERM_LJ = range(6)
TERM_NAMES = {"bond": TERM_BOND, "angle": TERM_ANGLE, "dihedral": TERM_DIHEDRAL,
              "exv": TERM_EXV, "dh": TERM_DH, "lj": TERM_LJ}

_i64p = C.POINTER(C.c_int64)
_f64p = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)


class OrcSpec(C.Structure):
    _fields_ = [
        ("n", C.c_int64), ("boundary", C.c_int32), ("single_molecule", C.c_int32),
        ("lower", C.c_double * 3), ("upper", C.c_double * 3),
        ("pos", _f64p), ("vel", _f64p), ("mass", _f64p),
        ("temperature", C.c_double), ("ionic_strength", C.c_double),
        ("ignore_molecule", C.c_int32), ("ignore_bond_within", C.c_int32),
        ("exv_on", C.c_int32), ("exv_eps", C.c_double), ("exv_cutoff", C.c_double),
        ("exv_margin", C.c_double), ("exv_n", C.c_int64), ("exv_idx", _i64p),
        ("exv_radius", _f64p),
        ("exv_kind", C.c_int32), ("exv_power", C.c_int32), ("exv_core", _f64p),
        ("dh_on", C.c_int32), ("dh_cutoff", C.c_double), ("dh_margin", C.c_double),
        ("dh_n", C.c_int64), ("dh_idx", _i64p), ("dh_charge", _f64p),
        ("lj_on", C.c_int32), ("lj_cutoff", C.c_double), ("lj_margin", C.c_double),
        ("lj_n", C.c_int64), ("lj_idx", _i64p), ("lj_sigma", _f64p), ("lj_eps", _f64p),
        ("lj_kind", C.c_int32),
        ("nbond", C.c_int64), ("bond_idx", _i64p), ("bond_k", _f64p), ("bond_v0", _f64p),
        ("nangle", C.c_int64), ("angle_idx", _i64p), ("angle_k", _f64p), ("angle_v0", _f64p),
        ("ndihd", C.c_int64), ("dihd_idx", _i64p), ("dihd_k", _f64p), ("dihd_n", _i32p),
        ("dihd_v0", _f64p),
        ("integrator", C.c_int32), ("dt", C.c_double), ("gamma", _f64p), ("seed", C.c_uint64),
    ]


def _ptr(a, ct):
    return a.ctypes.data_as(C.POINTER(ct)) if a is not None else None


LJ_KINDS = {"LennardJones": 0, "WCA": 1, "LennardJonesAttractive": 2, "UniformLennardJones": 3}
EXV_KINDS = {"ExcludedVolume": 0, "InversePower": 1, "HardCoreExcludedVolume": 2}


def _uniform_ignore(desc):
    """The oracle takes one ignore rule for all pair terms, with exclusions
    along "bond" connections only, and the default topology kinds of the
    local terms; anything else is outside what it restates."""
    rules = set()
    for t in desc.pair_terms():
        mol = t.ignore_molecule if getattr(t, "ignore_molecule", None) is not None else desc.ignore_molecule
        w = getattr(t, "ignore_within", None)
        if w is None:
            w = {"bond": desc.ignore_bond_within} if desc.ignore_bond_within > 0 else {}
        w = {k: int(v) for k, v in w.items() if int(v) > 0}
        if set(w) - {"bond"}:
            raise NotImplementedError("the oracle excludes along \"bond\" connections only")
        rules.add((mol, w.get("bond", 0)))
    if len(rules) > 1:
        raise NotImplementedError("the oracle takes one ignore rule for every pair term")
    kinds = (getattr(desc, "bond_topology", "bond"), getattr(desc, "angle_topology", "none"),
             getattr(desc, "dihedral_topology", "none"))
    if kinds != ("bond", "none", "none"):
        raise NotImplementedError("the oracle writes bonds as \"bond\" and angles, dihedrals as \"none\"")
    return rules.pop() if rules else (desc.ignore_molecule, int(desc.ignore_bond_within))


def make_spec(desc):
    """Returns (OrcSpec, keepalive) for a SystemDesc-like object."""
    keep = []

    def arr(x, dt):
        if x is None:
            return None
        a = np.ascontiguousarray(np.asarray(x, dtype=dt))
        keep.append(a)
        return a

    s = OrcSpec()
    s.n = desc.n
    s.boundary = 1 if desc.periodic else 0
    s.single_molecule = 1 if desc.single_molecule else 0
    s.lower = (C.c_double * 3)(*desc.lower)
    s.upper = (C.c_double * 3)(*desc.upper)
    s.pos = _ptr(arr(desc.pos, np.float64), C.c_double)
    s.vel = _ptr(arr(desc.vel, np.float64), C.c_double)
    s.mass = _ptr(arr(desc.mass, np.float64), C.c_double)
    s.temperature = desc.temperature
    s.ionic_strength = desc.ionic_strength
    mol, within = _uniform_ignore(desc)
    s.ignore_molecule = {"Nothing": 0, "Self": 1, "Intra": 1, "Others": 2, "Inter": 2}[mol]
    s.ignore_bond_within = within
    if desc.exv is not None:
        t = desc.exv
        s.exv_on, s.exv_eps, s.exv_cutoff, s.exv_margin = 1, t.epsilon, t.cutoff, t.margin
        s.exv_n = len(t.idx)
        s.exv_idx = _ptr(arr(t.idx, np.int64), C.c_int64)
        s.exv_radius = _ptr(arr(t.param0, np.float64), C.c_double)
        s.exv_kind = EXV_KINDS[t.kind]
        s.exv_power = int(t.exponent)
        if t.kind == "HardCoreExcludedVolume":
            s.exv_core = _ptr(arr(t.param1, np.float64), C.c_double)
    if desc.dh is not None:
        t = desc.dh
        s.dh_on, s.dh_cutoff, s.dh_margin = 1, t.cutoff, t.margin
        s.dh_n = len(t.idx)
        s.dh_idx = _ptr(arr(t.idx, np.int64), C.c_int64)
        s.dh_charge = _ptr(arr(t.param0, np.float64), C.c_double)
    if desc.lj is not None:
        t = desc.lj
        s.lj_on, s.lj_cutoff, s.lj_margin = 1, t.cutoff, t.margin
        s.lj_n = len(t.idx)
        s.lj_idx = _ptr(arr(t.idx, np.int64), C.c_int64)
        s.lj_sigma = _ptr(arr(t.param0, np.float64), C.c_double)
        s.lj_eps = _ptr(arr(t.param1, np.float64), C.c_double)
        s.lj_kind = LJ_KINDS[t.kind]
    if desc.bonds is not None:
        idx, k, v0 = desc.bonds
        s.nbond = len(idx)
        s.bond_idx = _ptr(arr(idx, np.int64), C.c_int64)
        s.bond_k = _ptr(arr(k, np.float64), C.c_double)
        s.bond_v0 = _ptr(arr(v0, np.float64), C.c_double)
    if desc.angles is not None:
        idx, k, v0 = desc.angles
        s.nangle = len(idx)
        s.angle_idx = _ptr(arr(idx, np.int64), C.c_int64)
        s.angle_k = _ptr(arr(k, np.float64), C.c_double)
        s.angle_v0 = _ptr(arr(v0, np.float64), C.c_double)
    if desc.dihedrals is not None:
        idx, k, nn, v0 = desc.dihedrals
        s.ndihd = len(idx)
        s.dihd_idx = _ptr(arr(idx, np.int64), C.c_int64)
        s.dihd_k = _ptr(arr(k, np.float64), C.c_double)
        s.dihd_n = _ptr(arr(nn, np.int32), C.c_int32)
        s.dihd_v0 = _ptr(arr(v0, np.float64), C.c_double)
    s.integrator = {"BAOAB": 0, "VelocityVerlet": 1, "UnderdampedLangevin": 2, "G-JFLangevin": 3,
                    "g-BAOABLangevin": 4}[desc.integrator]
    s.dt = desc.dt
    gam = desc.gamma if desc.gamma is not None else np.zeros(desc.n)
    s.gamma = _ptr(arr(gam, np.float64), C.c_double)
    s.seed = int(desc.seed)
    return s, keep


def build(reference_root: str | None = None) -> None:
    """Compiles liboracle.so and, when `reference_root` (the root of the
    reference tree; default: the environment variable MJOLNIR_REFERENCE_ROOT)
    names a tree that exists, the reference driver into _ref/."""
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True, env=env)
    ref = reference_root or os.environ.get("MJOLNIR_REFERENCE_ROOT")
    if ref and os.path.isdir(os.path.join(ref, "mjolnir")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFERENCE={ref}"], check=True, env=env)


# --------------------------------------------------------------------------
_olib = None


def _oracle_lib():
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        lib = C.CDLL(ORACLE_SO)
        lib.orc_create.restype = C.c_void_p
        lib.orc_create.argtypes = [C.POINTER(OrcSpec)]
        lib.orc_destroy.argtypes = [C.c_void_p]
        lib.orc_neighbors.restype = C.c_int64
        lib.orc_neighbors.argtypes = [C.c_void_p, C.c_int, _f64p, _i64p, C.c_int64]
        lib.orc_term_force.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p, _f64p]
        lib.orc_term_energy.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p]
        lib.orc_init_dynamics.argtypes = [C.c_void_p]
        lib.orc_run.argtypes = [C.c_void_p, C.c_int64]
        lib.orc_set_temperature.argtypes = [C.c_void_p, C.c_double]
        lib.orc_get_state.argtypes = [C.c_void_p, _f64p, _f64p, _f64p]
        lib.orc_rebuild_count.restype = C.c_int64
        lib.orc_rebuild_count.argtypes = [C.c_void_p, C.c_int]
        lib.orc_gaussian3.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, _f64p]
        lib.orc_philox4x32.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                       C.POINTER(C.c_uint32)]
        lib.orc_dh_params.argtypes = [C.c_double, C.c_double, C.c_double, _f64p]
        lib.orc_units.argtypes = [_f64p, _f64p, _f64p, _f64p]
        lib.orc_molecules.argtypes = [C.c_void_p, _i64p]
        lib.orc_exclusions.restype = C.c_int64
        lib.orc_exclusions.argtypes = [C.c_void_p, _i64p, _i64p, C.c_int64]
        _olib = lib
    return _olib


def _term(t):
    return TERM_NAMES[t] if isinstance(t, str) else int(t)


class _Common:
    n: int

    def _pairs(self, fn, term, *args):
        cnt = fn(self._h, _term(term), *args, None, 0)
        if cnt < 0:
            raise RuntimeError(f"term {term} not present ({cnt})")
        out = np.empty((max(cnt, 1), 2), dtype=np.int64)
        got = fn(self._h, _term(term), *args, _ptr(out, C.c_int64), cnt)
        assert got == cnt
        return out[:cnt]


class Oracle(_Common):
    """Plain-C restatement (oracle.c)."""

    def __init__(self, desc):
        self.lib = _oracle_lib()
        self._spec, self._keep = make_spec(desc)
        self.n = desc.n
        self._h = self.lib.orc_create(C.byref(self._spec))
        if not self._h:
            raise RuntimeError("orc_create failed")

    def close(self):
        if self._h:
            self.lib.orc_destroy(self._h)
            self._h = None

    __del__ = close

    def neighbors(self, term, pos=None):
        p = None if pos is None else np.ascontiguousarray(pos, dtype=np.float64)
        cnt = self.lib.orc_neighbors(self._h, _term(term), _ptr(p, C.c_double), None, 0)
        if cnt < 0:
            raise RuntimeError(f"term {term} not present")
        out = np.empty((max(cnt, 1), 2), dtype=np.int64)
        self.lib.orc_neighbors(self._h, _term(term), _ptr(p, C.c_double), _ptr(out, C.c_int64), cnt)
        return out[:cnt]

    def term_force(self, term, pos):
        p = np.ascontiguousarray(pos, dtype=np.float64)
        f = np.zeros((self.n, 3))
        e = C.c_double(0)
        if self.lib.orc_term_force(self._h, _term(term), _ptr(p, C.c_double), _ptr(f, C.c_double), C.byref(e)):
            raise RuntimeError(f"term {term} not present")
        return f, e.value

    def term_energy(self, term, pos):
        p = np.ascontiguousarray(pos, dtype=np.float64)
        e = C.c_double(0)
        if self.lib.orc_term_energy(self._h, _term(term), _ptr(p, C.c_double), C.byref(e)):
            raise RuntimeError(f"term {term} not present")
        return e.value

    def init_dynamics(self):
        self.lib.orc_init_dynamics(self._h)

    def run(self, nsteps):
        self.lib.orc_run(self._h, int(nsteps))

    def set_temperature(self, T):
        self.lib.orc_set_temperature(self._h, float(T))

    def state(self):
        p, v, f = (np.empty((self.n, 3)) for _ in range(3))
        self.lib.orc_get_state(self._h, _ptr(p, C.c_double), _ptr(v, C.c_double), _ptr(f, C.c_double))
        return p, v, f

    def rebuilds(self, term):
        return self.lib.orc_rebuild_count(self._h, _term(term))

    def molecules(self):
        m = np.empty(self.n, dtype=np.int64)
        self.lib.orc_molecules(self._h, _ptr(m, C.c_int64))
        return m

    def exclusions(self):
        r = np.empty(self.n + 1, dtype=np.int64)
        tot = self.lib.orc_exclusions(self._h, _ptr(r, C.c_int64), None, 0)
        idx = np.empty(max(tot, 1), dtype=np.int64)
        self.lib.orc_exclusions(self._h, _ptr(r, C.c_int64), _ptr(idx, C.c_int64), tot)
        return r, idx[:tot]


def gaussian3(seed, particle, step):
    out = np.empty(3)
    _oracle_lib().orc_gaussian3(seed, particle, step, _ptr(out, C.c_double))
    return out


def philox4x32(ctr, key):
    lib = _oracle_lib()
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib.orc_philox4x32(c, k, o)
    return list(o)


def dh_params(T, I, cutoff_ratio):
    out = np.empty(5)
    _oracle_lib().orc_dh_params(T, I, cutoff_ratio, _ptr(out, C.c_double))
    return out


def units():
    v = [C.c_double() for _ in range(4)]
    _oracle_lib().orc_units(*[C.byref(x) for x in v])
    return tuple(x.value for x in v)


# --------------------------------------------------------------------------
_rlib = None


def reference_available() -> bool:
    return os.path.exists(REF_SO)


def _ref_lib():
    global _rlib
    if _rlib is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO + " (the reference tree was not available at build time)")
        lib = C.CDLL(REF_SO)
        lib.ref_create.restype = C.c_void_p
        lib.ref_create.argtypes = [C.POINTER(OrcSpec), C.c_int]
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_destroy.argtypes = [C.c_void_p]
        lib.ref_term_force.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p]
        lib.ref_term_energy.argtypes = [C.c_void_p, C.c_int, _f64p]
        lib.ref_neighbors.restype = C.c_longlong
        lib.ref_neighbors.argtypes = [C.c_void_p, C.c_int, _i64p, C.c_longlong]
        lib.ref_initialize.argtypes = [C.c_void_p]
        lib.ref_run.restype = C.c_double
        lib.ref_run.argtypes = [C.c_void_p, C.c_longlong]
        lib.ref_get_state.argtypes = [C.c_void_p, _f64p, _f64p, _f64p]
        lib.ref_total_force.argtypes = [C.c_void_p, _f64p]
        lib.ref_total_energy.restype = C.c_double
        lib.ref_total_energy.argtypes = [C.c_void_p]
        lib.ref_max_threads.restype = C.c_int
        lib.ref_save_msgpack.restype = C.c_int
        lib.ref_save_msgpack.argtypes = [C.c_void_p, C.c_char_p]
        lib.ref_observe.restype = C.c_int
        lib.ref_observe.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_longlong, C.c_longlong,
                                    C.c_double]
        lib.ref_load_msgpack.restype = C.c_longlong
        lib.ref_load_msgpack.argtypes = [C.c_char_p, C.c_int, C.c_longlong, _f64p, _f64p, _f64p, _f64p,
                                         _f64p, _f64p, _f64p, _f64p]
        _rlib = lib
    return _rlib


class Reference(_Common):
    """The reference's own implementation (SimulatorTraits when parallel=False,
    OpenMPSimulatorTraits when parallel=True)."""

    def __init__(self, desc, parallel: bool = False):
        self.lib = _ref_lib()
        self._spec, self._keep = make_spec(desc)
        self.n = desc.n
        self._h = self.lib.ref_create(C.byref(self._spec), 1 if parallel else 0)
        if not self._h:
            raise RuntimeError("ref_create: " + self.lib.ref_last_error().decode())

    def close(self):
        if getattr(self, "_h", None):
            self.lib.ref_destroy(self._h)
            self._h = None

    __del__ = close

    def neighbors(self, term):
        cnt = self.lib.ref_neighbors(self._h, _term(term), None, 0)
        if cnt < 0:
            raise RuntimeError(f"term {term} not present")
        out = np.empty((max(cnt, 1), 2), dtype=np.int64)
        self.lib.ref_neighbors(self._h, _term(term), _ptr(out, C.c_int64), cnt)
        return out[:cnt]

    def term_force(self, term):
        f = np.zeros((self.n, 3))
        e = C.c_double(0)
        if self.lib.ref_term_force(self._h, _term(term), _ptr(f, C.c_double), C.byref(e)):
            raise RuntimeError(f"term {term} not present")
        return f, e.value

    def term_energy(self, term):
        e = C.c_double(0)
        if self.lib.ref_term_energy(self._h, _term(term), C.byref(e)):
            raise RuntimeError(f"term {term} not present")
        return e.value

    def initialize(self):
        self.lib.ref_initialize(self._h)

    def run(self, nsteps) -> float:
        return self.lib.ref_run(self._h, int(nsteps))

    def state(self):
        p, v, f = (np.empty((self.n, 3)) for _ in range(3))
        self.lib.ref_get_state(self._h, _ptr(p, C.c_double), _ptr(v, C.c_double), _ptr(f, C.c_double))
        return p, v, f

    def total_force(self):
        f = np.empty((self.n, 3))
        self.lib.ref_total_force(self._h, _ptr(f, C.c_double))
        return f

    def total_energy(self):
        return self.lib.ref_total_energy(self._h)

    def save_msgpack(self, prefix: str):
        """The reference's MsgPackSaver on the current state: writes
        prefix + "_system.msg"."""
        if self.lib.ref_save_msgpack(self._h, prefix.encode()):
            raise RuntimeError("ref_save_msgpack: " + self.lib.ref_last_error().decode())

    def observe(self, prefix: str, formats, total_step: int, save_step: int, dt: float):
        """Runs total_step steps as MolecularDynamicsSimulator does, with the
        reference's own observers of `formats` ("xyz", "dcd", "trr") and the
        energy observer writing under `prefix` (call initialize() first)."""
        mask = sum({"xyz": 1, "dcd": 2, "trr": 4}[f] for f in formats)
        if self.lib.ref_observe(self._h, prefix.encode(), mask, total_step, save_step, dt):
            raise RuntimeError("ref_observe: " + self.lib.ref_last_error().decode())

    @staticmethod
    def load_msgpack(path: str, periodic: bool, n_max: int = 1 << 22) -> dict:
        """The reference's MsgPackLoader::load_system on a file."""
        lib = _ref_lib()
        pos, vel, force = (np.empty((n_max, 3)) for _ in range(3))
        mass = np.empty(n_max)
        lo, up = np.zeros(3), np.zeros(3)
        t, i = C.c_double(0), C.c_double(0)
        n = lib.ref_load_msgpack(path.encode(), 1 if periodic else 0, n_max, _ptr(pos, C.c_double),
                                 _ptr(vel, C.c_double), _ptr(force, C.c_double), _ptr(mass, C.c_double),
                                 _ptr(lo, C.c_double), _ptr(up, C.c_double), C.byref(t), C.byref(i))
        if n < 0:
            raise RuntimeError("ref_load_msgpack: " + lib.ref_last_error().decode())
        return {"pos": pos[:n], "vel": vel[:n], "force": force[:n], "mass": mass[:n], "lower": lo,
                "upper": up, "temperature": t.value, "ionic_strength": i.value}

    @staticmethod
    def max_threads():
        return _ref_lib().ref_max_threads()


def synthetic_library():
    """The seeded input builders (``mjg_synth_*`` of
    include/mjolnir_b200_synthetic.h) as compiled into the reference driver,
    so that the reference arm of bench.py builds the benchmark's systems
    without loading the product library.  The same source file is compiled
    into both libraries, so the systems are identical."""
    lib = _ref_lib()
    for name in ("mjg_synth_polymer_chains", "mjg_synth_uniform_fluid"):
        getattr(lib, name).restype = C.c_int
    lib.mjg_synth_polymer_chains.argtypes = [C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double,
                                             C.c_uint64, _f64p]
    lib.mjg_synth_uniform_fluid.argtypes = [C.c_int64, C.c_double, C.c_double, C.c_uint64, _f64p]
    return lib
