"""Runs a Mjolnir input file on the GPU.

    python -m mjolnir_b200 input.toml [--precision fp64|mixed] [--device 0]

Reads the file with :func:`mjolnir_b200.input.load`, advances the system
``total_step`` steps and writes what the reference's simulator writes for the
same input, in the same layouts (:mod:`mjolnir_b200.observers`): at step 0,
every ``save_step`` steps and at the end, ``<path><prefix>.ene`` (energies of
the interactions in the order bonds, angles, dihedrals, then the global
terms; kinetic energy; the system's attributes) and the trajectory formats of
``files.output.format`` (xyz, dcd, trr); at step 0, every ``checkpoint_step``
steps and at the end, ``<prefix>_system.msg`` and ``<prefix>_rng.msg``
(:mod:`mjolnir_b200.checkpoint`).  The order of those calls is the one of
core/MolecularDynamicsSimulator.hpp:72-125 and
core/SimulatedAnnealingSimulator.hpp:121-150: observers and checkpoint before
the step, the temperature update of an annealing run after it.  The frames
are formatted and written on a second thread, in order, while the GPU runs
the next chunk.
``precision = "double"`` in the input selects the FP64 form unless
``--precision`` says otherwise (and sets the real type of the .trr file).
"""
from __future__ import annotations

import argparse
import os
import queue
import sys
import threading
import time

import numpy as np

from . import checkpoint
from . import observers as O
from .anneal import current
from .engine import Engine
from .input import load

# interaction names as the reference's name() returns them (the energy file's
# column titles): forcefield/local/*Interaction.hpp, GlobalPair*Interaction.hpp
PAIR_NAME = {"ExcludedVolume": "GlobalPairExcludedVolume", "LennardJones": "GlobalPairLennardJones",
             "DebyeHuckel": "Pair:DebyeHuckel", "WCA": "Pair:WCA",
             "LennardJonesAttractive": "Pair:LennardJonesAttractive",
             "UniformLennardJones": "Pair:LennardJones", "InversePower": "Pair:InversePower",
             "HardCoreExcludedVolume": "Pair:HardCoreExcludedVolume"}


def present_terms(desc):
    """(term key, column title) of every interaction, local then global."""
    out = []
    if desc.bonds is not None:
        out.append(("bond", "BondLength:Harmonic"))
    if desc.angles is not None:
        out.append(("angle", "BondAngle:Harmonic"))
    if desc.dihedrals is not None:
        out.append(("dihedral", "DihedralAngle:Cosine"))
    for key in ("exv", "dh", "lj"):
        t = getattr(desc, key)
        if t is not None:
            out.append((key, PAIR_NAME[t.kind]))
    return out


class _Writer:
    """Writes the observers' frames on a thread of its own, in order, while
    the GPU runs the next chunk; at most `depth` frames wait.  An error in
    the writer is raised at the next call."""

    def __init__(self, observers, dt, depth=2):
        self.obs, self.dt = observers, dt
        self.q = queue.Queue(maxsize=depth)
        self.err = None
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _run(self):
        while True:
            item = self.q.get()
            if item is None:
                return
            if self.err is None:
                try:
                    for o in self.obs:
                        o.output(item[0], self.dt, item[1])
                except Exception as e:          # re-raised in the caller's thread
                    self.err = e

    def put(self, step, frame):
        if self.err is not None:
            raise self.err
        self.q.put((step, frame))

    def close(self):
        self.q.put(None)
        self.t.join()
        if self.err is not None:
            raise self.err


def run(path: str, precision=None, device: int = 0, steps=None, out=sys.stderr) -> dict:
    inp = load(path)
    d = inp.desc
    prec = precision or ("fp64" if inp.precision == "double" else "mixed")
    total = inp.total_step if steps is None else int(steps)
    save = max(1, inp.save_step)
    ckpt = max(1, inp.checkpoint_step or save)
    prefix = inp.file_prefix
    if inp.output_path:
        os.makedirs(inp.output_path, exist_ok=True)
    terms = present_terms(d)
    attrs = dict(inp.attributes or {})
    if inp.schedule:                         # the schedule's first temperature, set at initialisation
        attrs["temperature"] = d.temperature
    eng = Engine(prec, device=device)
    sid = eng.add_system(d)
    eng.commit()
    width = tuple(float(u - lo) for u, lo in zip(d.upper, d.lower))
    molecules = eng.molecule_count(sid)

    def frame():
        p, v, f = eng.state(sid)
        e = eng.energies(sid)
        return O.Frame(pos=p, vel=v, force=f, mass=d.mass, energies=[(title, e[key]) for key, title in terms],
                       attributes=dict(attrs), names=inp.names, periodic=d.periodic, width=width,
                       molecules=molecules)

    def save_checkpoint():
        checkpoint.save(eng, sid, d, prefix, attributes=attrs, names=inp.names, groups=inp.groups)

    obs = O.make(inp.output_formats, prefix, real="f8" if inp.precision == "double" else "f4")
    t0 = time.perf_counter()
    anneal = inp.schedule                    # SimulatedAnnealing: (first, last, each_step)
    r_total = 1.0 / total if total else 0.0
    fr = frame()
    for o in obs:
        o.initialize(total, save, d.dt, fr)
    writer = _Writer(obs, d.dt)             # frames are formatted and written while the GPU steps
    done = 0
    try:
        while done < total:
            if done % save == 0:
                writer.put(done, frame())
            if done % ckpt == 0:
                save_checkpoint()
            k = min(save - done % save, ckpt - done % ckpt, total - done)
            if anneal:
                k = min(k, anneal[2] - done % anneal[2])
            eng.step(k)
            done += k
            if anneal and done % anneal[2] == 0:    # core/SimulatedAnnealingSimulator.hpp:144-154
                attrs["temperature"] = current(anneal[0], anneal[1], done * r_total)
                eng.set_temperature(sid, attrs["temperature"])
        fr = frame()                         # finalize: the last frame, then the checkpoint
        writer.put(total, fr)
    finally:
        writer.close()                       # frames already queued are written, even on an error
    for o in obs:
        o.finalize(total, d.dt, fr)
    save_checkpoint()
    wall = time.perf_counter() - t0
    eng.close()
    res = {"steps": total, "particles": d.n, "precision": prec, "wall_s": wall,
           "energy_file": prefix + ".ene", "formats": list(inp.output_formats)}
    if "xyz" in inp.output_formats:
        res["trajectory"] = prefix + "_position.xyz"
        res["velocities"] = prefix + "_velocity.xyz"
    if "dcd" in inp.output_formats:
        res["dcd"] = prefix + "_position.dcd"
    if "trr" in inp.output_formats:
        res["trr"] = prefix + ".trr"
    print(res, file=out)
    return res


def main():
    ap = argparse.ArgumentParser(prog="python -m mjolnir_b200")
    ap.add_argument("input")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default=None)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--steps", type=int, default=None, help="override total_step")
    a = ap.parse_args()
    run(a.input, a.precision, a.device, a.steps)


if __name__ == "__main__":
    main()
