"""Runs a Mjolnir input file on the GPU.

    python -m mjolnir_b200 input.toml [--precision fp64|mixed] [--device 0]

Reads the file with :func:`mjolnir_b200.input.load`, advances the system
``total_step`` steps and, every ``save_step`` steps (and at step 0), appends
the per-term energies, the kinetic energy and the attributes to
``<path>/<prefix>.ene``, and frames of positions and velocities to
``<path>/<prefix>_position.xyz`` and ``_velocity.xyz``, in the layout of the reference's
EnergyObserver and XYZObserver (core/EnergyObserver.hpp:63-153,
core/XYZObserver.hpp:46-76; interactions in the order bonds, angles,
dihedrals, then the global terms).  Every ``checkpoint_step`` steps and at the
end it writes ``<prefix>_system.msg`` and ``<prefix>_rng.msg``
(:mod:`mjolnir_b200.checkpoint`).
``precision = "double"`` in the input selects the FP64 form unless
``--precision`` says otherwise.  A ``SimulatedAnnealing`` input follows its
linear temperature schedule (:mod:`mjolnir_b200.anneal`).
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

from . import checkpoint
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


def _present(desc):
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


def _frame(f, names, arr, step):
    """One frame of core/XYZObserver.hpp:46-76: count, "step = N", then
    "name x y z" with eight decimals."""
    f.write(f"{arr.shape[0]}\nstep = {step}\n")
    f.write("".join(f"{nm} {x:.8f} {y:.8f} {z:.8f}\n" for nm, (x, y, z) in zip(names, arr)))


def run(path: str, precision=None, device: int = 0, steps=None, out=sys.stderr) -> dict:
    inp = load(path)
    d = inp.desc
    prec = precision or ("fp64" if inp.precision == "double" else "mixed")
    total = inp.total_step if steps is None else int(steps)
    save = max(1, inp.save_step)
    os.makedirs(inp.output_path, exist_ok=True)
    ene_path = os.path.join(inp.output_path, inp.output_prefix + ".ene")
    xyz_path = os.path.join(inp.output_path, inp.output_prefix + "_position.xyz")
    vel_path = os.path.join(inp.output_path, inp.output_prefix + "_velocity.xyz")
    terms = _present(d)
    widths = [max(len(title), 10) for _, title in terms]       # LocalForceField.hpp:57
    ckpt = max(1, inp.checkpoint_step or save)
    ck_prefix = os.path.join(inp.output_path, inp.output_prefix)
    names = ["X"] * d.n
    eng = Engine(prec, device=device)
    sid = eng.add_system(d)
    eng.commit()
    t0 = time.perf_counter()
    anneal = inp.schedule                    # SimulatedAnnealing: (first, last, each_step)
    r_total = 1.0 / total if total else 0.0
    temperature = d.temperature
    with open(ene_path, "w") as ene, open(xyz_path, "w") as xyz, open(vel_path, "w") as vel:
        # core/EnergyObserver.hpp:63-87 (header), :89-153 (rows)
        attrs = sorted({"temperature": 0.0, "ionic_strength": 0.0})
        ene.write("# timestep  " + "".join(title + " " for _, title in terms) + " kinetic_energy" +
                  "".join(f" attribute:{a}" for a in attrs) + "\n")
        done = 0
        while True:
            if done > 0 and (done % ckpt == 0 or done >= total):   # MsgPackSaver at checkpoint_step and at the end
                checkpoint.save(eng, sid, d, ck_prefix)
            if done % save == 0 or done >= total:
                e = eng.energies(sid)
                p, v, _ = eng.state(sid)
                kin = 0.5 * float(np.sum(np.sum(v * v, axis=1) * d.mass))
                values = {"temperature": temperature, "ionic_strength": d.ionic_strength}
                ene.write(f"{str(done):<11} " +
                          "".join(f"{e[key]:>{w}.6f} " for (key, _), w in zip(terms, widths)) +
                          f"{kin:>14.6f}" + "".join(f" {values[a]:>{10 + len(a)}.6f}" for a in attrs) + "\n")
                _frame(xyz, names, p, done)
                _frame(vel, names, v, done)
            if done >= total:
                break
            k = min(save - done % save, ckpt - done % ckpt, total - done)
            if anneal:
                k = min(k, anneal[2] - done % anneal[2])
            eng.step(k)
            done += k
            if anneal and done % anneal[2] == 0:    # core/SimulatedAnnealingSimulator.hpp:144-154
                temperature = current(anneal[0], anneal[1], done * r_total)
                eng.set_temperature(sid, temperature)
    wall = time.perf_counter() - t0
    eng.close()
    res = {"steps": total, "particles": d.n, "precision": prec, "wall_s": wall,
           "energy_file": ene_path, "trajectory": xyz_path, "velocities": vel_path}
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
