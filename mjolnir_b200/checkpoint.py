"""Checkpoints in the reference's MsgPack layout.

``<prefix>_system.msg`` is the map that core/MsgPackSaver.hpp:14-47 writes
and core/MsgPackLoader.hpp:91-... reads, in the same order and with the same
encodings (float64 reals, names and groups as strings)::

    {"boundary": nil | {"lower": [x, y, z], "upper": [x, y, z]},
     "particles": [{"mass", "position", "velocity", "force", "name", "group"}, ...],
     "virial": [9 reals], "attributes": {name: real, ... (sorted)},
     "dynamic_variables": {}}

so a file written here restarts the reference (``[[systems]] file_name =
"x_system.msg"``, input/read_system.hpp:105-131) and a file the reference
wrote restarts this library (:func:`mjolnir_b200.input.load` accepts the same
key).  The noise state is different: the reference stores its mt19937
state in ``<prefix>_rng.msg``; here the Langevin noise is Philox keyed by
(seed, particle, step), so ``<prefix>_rng.msg`` holds
``{"internal_state": "philox4x32-10 <seed> <step>"}``, which only this
library reads.
"""
from __future__ import annotations

import msgpack
import numpy as np

from .systems import SystemDesc

_KEYS = ("boundary", "particles", "virial", "attributes", "dynamic_variables")
_PKEYS = ("mass", "position", "velocity", "force", "name", "group")


class CheckpointError(ValueError):
    pass


def system_bytes(pos, vel, force, mass, periodic: bool, lower=None, upper=None,
                 attributes=None, names=None, groups=None) -> bytes:
    """The encoded ``_system.msg`` content."""
    pos, vel, force = (np.asarray(x, dtype=np.float64).reshape(-1, 3) for x in (pos, vel, force))
    mass = np.asarray(mass, dtype=np.float64).reshape(-1)
    n = pos.shape[0]
    boundary = ({"lower": [float(x) for x in lower], "upper": [float(x) for x in upper]}
                if periodic else None)
    P, V, F, M = pos.tolist(), vel.tolist(), force.tolist(), mass.tolist()
    particles = [{"mass": M[i], "position": P[i], "velocity": V[i], "force": F[i],
                  "name": names[i] if names is not None else "X",
                  "group": groups[i] if groups is not None else "NONE"} for i in range(n)]
    attrs = {k: float(v) for k, v in sorted((attributes or {}).items())}   # std::map order
    root = {"boundary": boundary, "particles": particles, "virial": [0.0] * 9,
            "attributes": attrs, "dynamic_variables": {}}
    return msgpack.packb(root, use_bin_type=True)


def write_system(path: str, *args, **kw):
    with open(path, "wb") as f:
        f.write(system_bytes(*args, **kw))


def read_system(path: str) -> dict:
    """Reads a ``_system.msg`` file (written here or by the reference)."""
    try:
        with open(path, "rb") as f:
            root = msgpack.unpackb(f.read(), raw=False, strict_map_key=False)
    except FileNotFoundError:
        raise CheckpointError(f"file not found: {path}") from None
    except (ValueError, msgpack.exceptions.ExtraData) as e:
        raise CheckpointError(f"{path}: not a MsgPack file ({e})") from None
    if not isinstance(root, dict) or tuple(root) != _KEYS:
        raise CheckpointError(f"{path}: the root must be a map with keys {_KEYS}")
    parts = root["particles"]
    if not parts or any(not isinstance(p, dict) or tuple(p) != _PKEYS for p in parts):
        raise CheckpointError(f"{path}: every particle must be a map with keys {_PKEYS}")
    b = root["boundary"]
    out = {
        "periodic": b is not None,
        "lower": tuple(b["lower"]) if b is not None else (0.0, 0.0, 0.0),
        "upper": tuple(b["upper"]) if b is not None else (0.0, 0.0, 0.0),
        "mass": np.array([p["mass"] for p in parts], dtype=np.float64),
        "pos": np.array([p["position"] for p in parts], dtype=np.float64),
        "vel": np.array([p["velocity"] for p in parts], dtype=np.float64),
        "force": np.array([p["force"] for p in parts], dtype=np.float64),
        "names": [p["name"] for p in parts],
        "groups": [p["group"] for p in parts],
        "attributes": dict(root["attributes"]),
    }
    if out["pos"].shape != (len(parts), 3):
        raise CheckpointError(f"{path}: positions must have 3 components")
    return out


def write_rng(path: str, seed: int, step: int):
    with open(path, "wb") as f:
        f.write(msgpack.packb({"internal_state": f"philox4x32-10 {int(seed)} {int(step)}"}))


def read_rng(path: str):
    """(seed, step) of a ``_rng.msg`` file written by :func:`write_rng`."""
    with open(path, "rb") as f:
        root = msgpack.unpackb(f.read(), raw=False)
    st = root.get("internal_state", "") if isinstance(root, dict) else ""
    parts = st.split()
    if len(parts) != 3 or parts[0] != "philox4x32-10":
        raise CheckpointError(f"{path}: not a Philox noise state (an mt19937 state of the reference "
                              "cannot continue this library's noise stream)")
    return int(parts[1]), int(parts[2])


def save(engine, sid: int, desc: SystemDesc, prefix: str, attributes=None, names=None, groups=None):
    """Writes ``<prefix>_system.msg`` and ``<prefix>_rng.msg`` for system
    `sid` of `engine` (its current state; `desc` gives masses and box;
    `attributes` default to the temperature and ionic strength of `desc`;
    names "X" and groups "NONE" unless given)."""
    pos, vel, force = engine.state(sid)
    if attributes is None:
        attributes = {"temperature": desc.temperature, "ionic_strength": desc.ionic_strength}
    write_system(prefix + "_system.msg", pos, vel, force, desc.mass, desc.periodic, desc.lower,
                 desc.upper, attributes, names, groups)
    write_rng(prefix + "_rng.msg", desc.seed, engine.step_count(sid))


def restore(prefix: str, desc: SystemDesc) -> SystemDesc:
    """`desc` with the state of a checkpoint (positions, velocities, noise
    step); the interactions are those of `desc`.  Add the result to an engine
    and the run continues where the checkpoint left it."""
    s = read_system(prefix + "_system.msg")
    if s["pos"].shape[0] != desc.n:
        raise CheckpointError(f"checkpoint has {s['pos'].shape[0]} particles, the system {desc.n}")
    out = desc.copy()
    out.pos = s["pos"]
    out.vel = s["vel"]
    seed, step = read_rng(prefix + "_rng.msg")
    if seed != desc.seed:
        raise CheckpointError("checkpoint seed differs from the system's")
    out.start_step = step
    return out
