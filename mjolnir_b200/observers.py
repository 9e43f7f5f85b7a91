"""Trajectory and energy writers in the reference's file layouts.

Each class follows one observer of the reference, with the same file names
under the same prefix (``<path><prefix>``) and the same bytes:

* :class:`EnergyObserver` -- ``<prefix>.ene`` (core/EnergyObserver.hpp:27-153);
* :class:`XYZObserver` -- ``<prefix>_position.xyz``, ``<prefix>_velocity.xyz``
  (core/XYZObserver.hpp:46-76);
* :class:`DCDObserver` -- ``<prefix>_position.dcd``, ``<prefix>_velocity.dcd``
  (core/DCDObserver.hpp:30-330), single-precision frames, the frame count
  patched into the header at ``finalize``;
* :class:`TRRObserver` -- ``<prefix>.trr`` (core/TRRObserver.hpp:33-230),
  positions, velocities and forces in the simulation's real type.

The one deliberate difference is the 80-byte title record of the DCD header,
which names this library instead of carrying the reference's text.

The call sequence is the one MolecularDynamicsSimulator makes
(core/MolecularDynamicsSimulator.hpp:72-125): ``initialize`` once, ``output``
at every step that is a multiple of ``save_step`` and once more at the end,
then ``finalize``.  Every call takes a :class:`Frame`, the host copy of one
system's state.
"""
from __future__ import annotations

import dataclasses
import struct
from typing import List, Optional, Sequence, Tuple

import numpy as np

DCD_TITLE = b"DCD written by mjolnir_b200 (Mjolnir-compatible trajectory)".ljust(80, b"\0")
assert len(DCD_TITLE) == 80


@dataclasses.dataclass
class Frame:
    """One system's state as the observers read it."""
    pos: np.ndarray                            # (n, 3) float64
    vel: np.ndarray                            # (n, 3) float64
    force: np.ndarray                          # (n, 3) float64
    mass: np.ndarray                           # (n,)
    energies: Sequence[Tuple[str, float]] = ()  # (interaction name, energy), force-field order
    attributes: Optional[dict] = None          # name -> value (written sorted, as std::map)
    names: Optional[Sequence[str]] = None      # particle names ("X" by default)
    periodic: bool = False
    width: Tuple[float, float, float] = (0.0, 0.0, 0.0)   # box edge lengths (periodic)
    molecules: int = 0                         # Topology::number_of_molecules

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])


def kinetic_energy(vel: np.ndarray, mass: np.ndarray) -> float:
    """EnergyObserver::calc_kinetic_energy (:155-168): sum of |v|^2 m in
    particle order, then halved (the same roundings: cumsum accumulates left
    to right)."""
    v = np.asarray(vel, dtype=np.float64)
    l2 = (v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2]
    terms = l2 * np.asarray(mass, dtype=np.float64)
    total = float(np.cumsum(terms)[-1]) if terms.size else 0.0
    return total * 0.5


def _clear(path: str):
    open(path, "w").close()


class EnergyObserver:
    def __init__(self, prefix: str, length_unit: str = "angstrom", energy_unit: str = "kcal/mol"):
        self.file_name = prefix + ".ene"
        self.length_unit, self.energy_unit = length_unit, energy_unit
        self.widths: List[int] = []
        _clear(self.file_name)

    def initialize(self, total_step: int, save_step: int, dt: float, frame: Frame):
        # :35-60; column widths max(len(name), 10) (LocalForceField.hpp:57,
        # GlobalForceField.hpp:57)
        self.widths = [max(len(name), 10) for name, _ in frame.energies]
        attrs = sorted((frame.attributes or {}).keys())
        with open(self.file_name, "a") as f:
            f.write(f"# unit of length : {self.length_unit}, unit of energy : {self.energy_unit}\n")
            f.write("# timestep  " + "".join(name + " " for name, _ in frame.energies) + " kinetic_energy" +
                    "".join(f" attribute:{a}" for a in attrs) + "\n")

    def output(self, step: int, dt: float, frame: Frame):
        # :89-153: step left in 11 columns, energies "%{w}.6f ", kinetic
        # "%14.6f", attributes " %{10 + len(name)}.6f"
        attrs = sorted((frame.attributes or {}).items())
        line = f"{str(step):<11} "
        line += "".join(f"{e:>{w}.6f} " for (_, e), w in zip(frame.energies, self.widths))
        line += f"{kinetic_energy(frame.vel, frame.mass):>14.6f}"
        line += "".join(f" {v:>{10 + len(a)}.6f}" for a, v in attrs)
        with open(self.file_name, "a") as f:
            f.write(line + "\n")

    def finalize(self, total_step: int, dt: float, frame: Frame):
        pass


class XYZObserver:
    def __init__(self, prefix: str):
        self.xyz_name = prefix + "_position.xyz"
        self.vel_name = prefix + "_velocity.xyz"
        _clear(self.xyz_name)
        _clear(self.vel_name)

    def initialize(self, total_step: int, save_step: int, dt: float, frame: Frame):
        pass

    @staticmethod
    def _frame(path, names, arr, step):
        with open(path, "a") as f:
            f.write(f"{arr.shape[0]}\nstep = {step}\n")
            f.write("".join(f"{nm} {x:.8f} {y:.8f} {z:.8f}\n" for nm, (x, y, z) in zip(names, arr.tolist())))

    def output(self, step: int, dt: float, frame: Frame):
        names = frame.names if frame.names is not None else ["X"] * frame.n
        self._frame(self.xyz_name, names, frame.pos, step)
        self._frame(self.vel_name, names, frame.vel, step)

    def finalize(self, total_step: int, dt: float, frame: Frame):
        pass


def _block(payload: bytes) -> bytes:
    """A Fortran unformatted record: int32 size, payload, int32 size."""
    n = struct.pack("<i", len(payload))
    return n + payload + n


class DCDObserver:
    def __init__(self, prefix: str):
        self.pos_name = prefix + "_position.dcd"
        self.vel_name = prefix + "_velocity.dcd"
        self.frames = 0
        _clear(self.pos_name)
        _clear(self.vel_name)

    def _header(self, total_step, save_step, dt, frame: Frame) -> bytes:
        # :118-180: CORD record (frames patched later, first index 0, save
        # interval, total steps, molecules, 4 zeros, dt as float, unit-cell
        # flag, 8 zeros, version 24), the title record, the particle count
        first = (b"CORD" + struct.pack("<9i", 0, 0, int(save_step), int(total_step), int(frame.molecules),
                                       0, 0, 0, 0) +
                 struct.pack("<f", dt) + struct.pack("<i", 1 if frame.periodic else 0) +
                 struct.pack("<8i", *([0] * 8)) + struct.pack("<i", 24))
        title = struct.pack("<i", 1) + DCD_TITLE
        return _block(first) + _block(title) + _block(struct.pack("<i", frame.n))

    def initialize(self, total_step: int, save_step: int, dt: float, frame: Frame):
        h = self._header(total_step, save_step, dt, frame)
        for path in (self.pos_name, self.vel_name):
            with open(path, "ab") as f:
                f.write(h)

    @staticmethod
    def _xyz_blocks(arr: np.ndarray) -> bytes:
        a = np.asarray(arr, dtype=np.float64).astype("<f4")
        return b"".join(_block(np.ascontiguousarray(a[:, k]).tobytes()) for k in range(3))

    def output(self, step: int, dt: float, frame: Frame):
        # :262-330.  The unit cell (A, gamma, B, beta, alpha, C; angles 90) goes
        # into the position file only, although both headers set the flag.
        self.frames += 1
        with open(self.pos_name, "ab") as f:
            if frame.periodic:
                A, B, Cw = (float(x) for x in frame.width)
                f.write(_block(struct.pack("<6d", A, 90.0, B, 90.0, 90.0, Cw)))
            f.write(self._xyz_blocks(frame.pos))
        with open(self.vel_name, "ab") as f:
            f.write(self._xyz_blocks(frame.vel))

    def finalize(self, total_step: int, dt: float, frame: Frame):
        # :71-96: the number of frames after the first record's size and "CORD"
        for path in (self.pos_name, self.vel_name):
            with open(path, "r+b") as f:
                f.seek(8)
                f.write(struct.pack("<i", self.frames))


class TRRObserver:
    def __init__(self, prefix: str, real: str = "f8"):
        """`real`: "f8" (double) or "f4" (float), the simulation's real type."""
        self.prefix = prefix
        self.trr_name = prefix + ".trr"
        self.real = np.dtype("<" + real)
        _clear(self.trr_name)

    def initialize(self, total_step: int, save_step: int, dt: float, frame: Frame):
        pass

    def output(self, step: int, dt: float, frame: Frame):
        # :151-224: magic 1993, 13, the title (its length, then the prefix
        # bytes), the record sizes (box, x, v, f), natoms, step, dt, lambda,
        # box vectors when periodic, then x, v, f
        rs = self.real.itemsize
        title = self.prefix.encode()
        crd = rs * 3 * frame.n
        box = rs * 9 if frame.periodic else 0
        head = struct.pack("<3i", 1993, 13, len(title)) + title
        head += struct.pack("<13i", 0, 0, box, 0, 0, 0, 0, crd, crd, crd, frame.n, int(step), 0)
        head += np.array([dt, 0.0], dtype=self.real).tobytes()
        out = [head]
        if frame.periodic:
            wx, wy, wz = (float(x) for x in frame.width)
            out.append(np.array([wx, 0, 0, 0, wy, 0, 0, 0, wz], dtype=self.real).tobytes())
        for arr in (frame.pos, frame.vel, frame.force):
            out.append(np.asarray(arr, dtype=np.float64).astype(self.real).tobytes())
        with open(self.trr_name, "ab") as f:
            f.write(b"".join(out))

    def finalize(self, total_step: int, dt: float, frame: Frame):
        pass


FORMATS = ("xyz", "dcd", "trr")


def make(formats: Sequence[str], prefix: str, real: str = "f8"):
    """The observers read_observer builds (input/read_observer.hpp:17-96): one
    per format, in order, then the energy observer."""
    obs = []
    for fmt in formats:
        if fmt == "xyz":
            obs.append(XYZObserver(prefix))
        elif fmt == "dcd":
            obs.append(DCDObserver(prefix))
        elif fmt == "trr":
            obs.append(TRRObserver(prefix, real))
        else:
            raise ValueError(f'output format "{fmt}" is not one of {FORMATS}')
    obs.append(EnergyObserver(prefix))
    return obs
