"""Python front end of the C ABI: an :class:`Engine` owns one device context
(one arena of resident systems) and advances every committed system together.

    eng = Engine(precision="mixed")
    sid = eng.add_system(desc)          # a systems.SystemDesc
    eng.commit()                        # lists + first forces on the GPU
    eng.step(1000)                      # BAOAB steps of every system
    pos, vel, force = eng.state(sid)

All work happens in libmjolnir_b200.so; this module only moves arguments.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as A
from .systems import SystemDesc


def _arr(x, dt):
    return np.ascontiguousarray(np.asarray(x, dtype=dt))


class Engine:
    def __init__(self, precision: str = "mixed", device: int = 0, graphs: bool = True,
                 rollback: bool = True):
        self.lib = A.lib()
        p = {"fp64": A.PRECISION_FP64, "mixed": A.PRECISION_MIXED}[precision]
        h = C.c_void_p()
        code = self.lib.mjg_context_create(device, p, C.byref(h))
        if code != A.OK:
            raise A.MjgError(code, "mjg_context_create failed (no usable CUDA device?)")
        self.ctx = h
        self.precision = precision
        self.n_of = {}
        A.check(self.ctx, self.lib.mjg_context_set_graphs(self.ctx, 1 if graphs else 0))
        A.check(self.ctx, self.lib.mjg_context_set_rollback(self.ctx, 1 if rollback else 0))

    def reserve(self, particles: int):
        """Page-locks the commit buffers for an arena of up to `particles`."""
        self._c(self.lib.mjg_context_reserve(self.ctx, int(particles)))

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.mjg_context_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _c(self, code):
        return A.check(self.ctx, code)

    # ------------------------------------------------------------ systems
    def add_system(self, d: SystemDesc) -> int:
        L = self.lib
        pos = _arr(d.pos, np.float64)
        vel = _arr(d.vel, np.float64)
        mass = _arr(d.mass, np.float64)
        lo = _arr(d.lower, np.float64)
        up = _arr(d.upper, np.float64)
        sid = C.c_int()
        self._c(L.mjg_system_create(self.ctx, d.n, A.PERIODIC_CUBOID if d.periodic else A.UNLIMITED,
                                    A.f64(lo), A.f64(up), A.f64(pos), A.f64(vel), A.f64(mass),
                                    C.byref(sid)))
        s = sid.value
        self.n_of[s] = d.n
        self._c(L.mjg_system_set_attributes(self.ctx, s, float(d.temperature), float(d.ionic_strength)))
        if d.single_molecule and d.n > 1:
            chain = np.stack([np.arange(d.n - 1), np.arange(1, d.n)], axis=1).astype(np.int64)
            chain = np.ascontiguousarray(chain)
            self._c(L.mjg_system_add_connections(self.ctx, s, b"bond", d.n - 1, A.i64(chain)))
        for term, t in ((A.TERM_EXV, d.exv), (A.TERM_DH, d.dh), (A.TERM_LJ, d.lj)):
            if t is None:
                continue
            ign = A.IGNORE[t.ignore_molecule if t.ignore_molecule is not None else d.ignore_molecule]
            if t.ignore_within is not None:
                within = [(k, int(v)) for k, v in t.ignore_within.items() if int(v) > 0]
            else:
                within = [("bond", d.ignore_bond_within)] if d.ignore_bond_within > 0 else []
            idx = _arr(t.idx, np.int64)
            p0 = _arr(t.param0, np.float64)
            if term == A.TERM_EXV and t.kind == "ExcludedVolume":
                self._c(L.mjg_exv_set(self.ctx, s, float(t.epsilon), float(t.cutoff), float(t.margin),
                                      len(idx), A.i64(idx), A.f64(p0)))
            elif term == A.TERM_EXV:                # InversePower, HardCoreExcludedVolume
                p1 = _arr(t.param1, np.float64) if t.param1 is not None else None
                self._c(L.mjg_exv_family_set(self.ctx, s, t.kind.encode(), float(t.epsilon), float(t.cutoff),
                                             int(t.exponent), float(t.margin), len(idx), A.i64(idx),
                                             A.f64(p0), A.f64(p1)))
            elif term == A.TERM_DH:
                self._c(L.mjg_dh_set(self.ctx, s, float(t.cutoff), float(t.margin), len(idx),
                                     A.i64(idx), A.f64(p0)))
            elif t.kind == "LennardJones":
                p1 = _arr(t.param1, np.float64)
                self._c(L.mjg_lj_set(self.ctx, s, float(t.cutoff), float(t.margin), len(idx),
                                     A.i64(idx), A.f64(p0), A.f64(p1)))
            else:                                   # WCA, LennardJonesAttractive, UniformLennardJones
                p1 = _arr(t.param1, np.float64)
                self._c(L.mjg_pair_set(self.ctx, s, t.kind.encode(), float(t.cutoff), float(t.margin),
                                       len(idx), A.i64(idx), A.f64(p0), A.f64(p1)))
            kinds = (C.c_char_p * max(1, len(within)))(*[k.encode() for k, _ in within])
            vals = _arr([w for _, w in within] or [0], np.int32)
            self._c(L.mjg_ignore_set(self.ctx, s, term, ign, len(within), kinds, A.i32(vals)))
        if d.bonds is not None:
            idx, k, v0 = (_arr(d.bonds[0], np.int64), _arr(d.bonds[1], np.float64), _arr(d.bonds[2], np.float64))
            self._c(L.mjg_bonds_set(self.ctx, s, d.bond_topology.encode(), len(k), A.i64(idx), A.f64(k), A.f64(v0)))
        if d.angles is not None:
            idx, k, v0 = (_arr(d.angles[0], np.int64), _arr(d.angles[1], np.float64), _arr(d.angles[2], np.float64))
            self._c(L.mjg_angles_set(self.ctx, s, d.angle_topology.encode(), len(k), A.i64(idx), A.f64(k), A.f64(v0)))
        if d.dihedrals is not None:
            idx = _arr(d.dihedrals[0], np.int64)
            k = _arr(d.dihedrals[1], np.float64)
            nn = _arr(d.dihedrals[2], np.int32)
            v0 = _arr(d.dihedrals[3], np.float64)
            self._c(L.mjg_dihedrals_set(self.ctx, s, d.dihedral_topology.encode(), len(k), A.i64(idx), A.f64(k), A.i32(nn), A.f64(v0)))
        kind = {"VelocityVerlet": A.VELOCITY_VERLET, "UnderdampedLangevin": A.UNDERDAMPED_LANGEVIN,
                "G-JFLangevin": A.GJF_LANGEVIN, "g-BAOABLangevin": A.GBAOAB_LANGEVIN}.get(d.integrator, A.BAOAB)
        gam = _arr(d.gamma if d.gamma is not None else np.zeros(d.n), np.float64)
        self._c(L.mjg_integrator_set(self.ctx, s, kind, float(d.dt), A.f64(gam), int(d.seed) & ((1 << 64) - 1)))
        if d.start_step:
            self._c(L.mjg_system_set_step(self.ctx, s, int(d.start_step)))
        return s

    def remove_system(self, sid: int):
        self._c(self.lib.mjg_system_remove(self.ctx, sid))
        self.n_of.pop(sid, None)

    def set_temperature(self, sid: int, temperature: float):
        """Langevin temperature from the next step on (simulated annealing)."""
        self._c(self.lib.mjg_system_set_temperature(self.ctx, sid, float(temperature)))

    def freeze(self, sid: int, frozen: bool = True):
        self._c(self.lib.mjg_system_freeze(self.ctx, sid, 1 if frozen else 0))

    def commit(self):
        self._c(self.lib.mjg_commit(self.ctx))

    def step(self, nsteps: int = 1):
        self._c(self.lib.mjg_step(self.ctx, int(nsteps)))

    def synchronize(self):
        self._c(self.lib.mjg_synchronize(self.ctx))

    def rebuild(self):
        self._c(self.lib.mjg_rebuild(self.ctx))

    # -------------------------------------------------------------- state
    def state(self, sid: int):
        n = self.n_of[sid]
        p, v, f = (np.empty((n, 3)) for _ in range(3))
        self._c(self.lib.mjg_get_state(self.ctx, sid, A.f64(p), A.f64(v), A.f64(f)))
        return p, v, f

    def positions(self, sid: int):
        n = self.n_of[sid]
        p = np.empty((n, 3))
        self._c(self.lib.mjg_get_state(self.ctx, sid, A.f64(p), None, None))
        return p

    def set_state(self, sid: int, pos=None, vel=None):
        p = None if pos is None else _arr(pos, np.float64)
        v = None if vel is None else _arr(vel, np.float64)
        self._c(self.lib.mjg_set_state(self.ctx, sid, A.f64(p), A.f64(v)))

    def total_particles(self) -> int:
        n = C.c_int64()
        self._c(self.lib.mjg_particle_count(self.ctx, -1, C.byref(n)))
        return n.value

    def get_state_all(self, pos_out=None, vel_out=None):
        self._c(self.lib.mjg_get_state_all(self.ctx, A.f64(pos_out), A.f64(vel_out)))

    def set_state_all(self, pos=None, vel=None):
        self._c(self.lib.mjg_set_state_all(self.ctx, A.f64(pos), A.f64(vel)))

    def energies(self, sid: int) -> dict:
        out = np.zeros(6)
        self._c(self.lib.mjg_energies(self.ctx, sid, A.f64(out)))
        return dict(zip(A.TERM_NAMES, out.tolist()))

    def term_force(self, sid: int, term):
        t = A.TERM_NAMES.index(term) if isinstance(term, str) else int(term)
        f = np.empty((self.n_of[sid], 3))
        e = C.c_double()
        self._c(self.lib.mjg_term_force(self.ctx, sid, t, A.f64(f), C.byref(e)))
        return f, e.value

    def neighbors(self, sid: int, term) -> np.ndarray:
        t = A.TERM_NAMES.index(term) if isinstance(term, str) else int(term)
        cnt = C.c_int64()
        self._c(self.lib.mjg_neighbors(self.ctx, sid, t, None, 0, C.byref(cnt)))
        out = np.empty((max(cnt.value, 1), 2), dtype=np.int64)
        self._c(self.lib.mjg_neighbors(self.ctx, sid, t, A.i64(out), cnt.value, C.byref(cnt)))
        return out[: cnt.value]

    def rebuild_count(self, sid: int, term) -> int:
        t = A.TERM_NAMES.index(term) if isinstance(term, str) else int(term)
        c = C.c_int64()
        self._c(self.lib.mjg_rebuild_count(self.ctx, sid, t, C.byref(c)))
        return c.value

    def step_count(self, sid: int) -> int:
        c = C.c_int64()
        self._c(self.lib.mjg_step_count(self.ctx, sid, C.byref(c)))
        return c.value

    def molecule_count(self, sid: int) -> int:
        """Molecules of a system (groups joined by "bond" connections)."""
        c = C.c_int64()
        self._c(self.lib.mjg_molecule_count(self.ctx, sid, C.byref(c)))
        return c.value

    def device_bytes(self) -> int:
        c = C.c_int64()
        self._c(self.lib.mjg_device_bytes(self.ctx, C.byref(c)))
        return c.value

    def pair_count(self, sid: int, term) -> int:
        """Interacting pairs (i < j inside the cutoff) of a global term; sid=-1: all systems."""
        t = A.TERM_NAMES.index(term) if isinstance(term, str) else int(term)
        c = C.c_int64()
        self._c(self.lib.mjg_pair_count(self.ctx, sid, t, C.byref(c)))
        return c.value

    def debug_set_list_capacity(self, term, cap: int):
        t = A.TERM_NAMES.index(term) if isinstance(term, str) else int(term)
        self._c(self.lib.mjg_set_list_capacity(self.ctx, t, int(cap)))

    def stream_handle(self) -> int:
        """cudaStream_t of the context, as an integer (for torch.cuda.ExternalStream)."""
        h = C.c_void_p()
        self._c(self.lib.mjg_context_get_stream(self.ctx, C.byref(h)))
        return h.value or 0

    def time_kernel(self, term, reps: int = 20) -> float:
        """Average ms per launch of a term's force kernel on the current lists."""
        t = A.TERM_NAMES.index(term) if isinstance(term, str) else int(term)
        ms = C.c_double()
        self._c(self.lib.mjg_time_kernel(self.ctx, t, int(reps), C.byref(ms)))
        return ms.value

    def set_threads_per_particle(self, term, tpp: int):
        t = A.TERM_NAMES.index(term) if isinstance(term, str) else int(term)
        self._c(self.lib.mjg_set_threads_per_particle(self.ctx, t, int(tpp)))

    def get_threads_per_particle(self, term) -> int:
        t = A.TERM_NAMES.index(term) if isinstance(term, str) else int(term)
        v = C.c_int()
        self._c(self.lib.mjg_get_threads_per_particle(self.ctx, t, C.byref(v)))
        if v.value == 0:
            raise A.MjgError(A.EINVAL, f"term {term} not present")
        return v.value

    def set_pair_unroll(self, term, unroll: int):
        t = A.TERM_NAMES.index(term) if isinstance(term, str) else int(term)
        self._c(self.lib.mjg_set_pair_unroll(self.ctx, t, int(unroll)))

    def get_pair_unroll(self, term) -> int:
        t = A.TERM_NAMES.index(term) if isinstance(term, str) else int(term)
        v = C.c_int()
        self._c(self.lib.mjg_get_pair_unroll(self.ctx, t, C.byref(v)))
        return v.value

    def set_pair_schedule(self, term, schedule: int):
        t = A.TERM_NAMES.index(term) if isinstance(term, str) else int(term)
        self._c(self.lib.mjg_set_pair_schedule(self.ctx, t, int(schedule)))

    def get_pair_schedule(self, term) -> int:
        t = A.TERM_NAMES.index(term) if isinstance(term, str) else int(term)
        v = C.c_int()
        self._c(self.lib.mjg_get_pair_schedule(self.ctx, t, C.byref(v)))
        return v.value

    def set_half_lists(self, term, on: bool):
        """Half Verlet lists for the term (mixed form only): each pair in one
        list, the partner's force added by the same evaluation; identical
        results, half the list words and pair evaluations."""
        t = A.TERM_NAMES.index(term) if isinstance(term, str) else int(term)
        self._c(self.lib.mjg_set_half_lists(self.ctx, t, int(bool(on))))

    def get_half_lists(self, term) -> bool:
        t = A.TERM_NAMES.index(term) if isinstance(term, str) else int(term)
        v = C.c_int()
        self._c(self.lib.mjg_get_half_lists(self.ctx, t, C.byref(v)))
        return bool(v.value)

    def set_build_lanes(self, term, lanes: int):
        """Lanes per particle of the term's list build (4, 8, 16 or 32)."""
        t = A.TERM_NAMES.index(term) if isinstance(term, str) else int(term)
        self._c(self.lib.mjg_set_build_lanes(self.ctx, t, int(lanes)))

    def get_build_lanes(self, term) -> int:
        t = A.TERM_NAMES.index(term) if isinstance(term, str) else int(term)
        v = C.c_int()
        self._c(self.lib.mjg_get_build_lanes(self.ctx, t, C.byref(v)))
        return v.value

    def set_margin(self, term, margin: float):
        t = A.TERM_NAMES.index(term) if isinstance(term, str) else int(term)
        self._c(self.lib.mjg_set_margin(self.ctx, t, float(margin)))

    def launch_count(self) -> int:
        c = C.c_int64()
        self._c(self.lib.mjg_launch_count(self.ctx, C.byref(c)))
        return c.value
