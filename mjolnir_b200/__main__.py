"""Runs a Mjolnir input file on the GPU.

    python -m mjolnir_b200 input.toml [--precision fp64|mixed] [--device 0]

Reads the file with :func:`mjolnir_b200.input.load`, advances the system
``total_step`` steps and, every ``save_step`` steps (and at step 0), appends
the per-term energies and the kinetic energy to ``<path>/<prefix>.ene`` and a
frame of positions to ``<path>/<prefix>.xyz`` (the quantities the reference's
EnergyObserver and XYZObserver write; core/EnergyObserver.hpp:89-153).
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

from .anneal import current
from .engine import Engine
from .input import load

TERM_LABEL = {"bond": "BondLength:Harmonic", "angle": "BondAngle:Harmonic",
              "dihedral": "DihedralAngle:Cosine", "exv": "ExcludedVolume",
              "dh": "DebyeHuckel", "lj": "LennardJones"}


def _present(desc):
    out = []
    if desc.bonds is not None:
        out.append("bond")
    if desc.angles is not None:
        out.append("angle")
    if desc.dihedrals is not None:
        out.append("dihedral")
    for key in ("exv", "dh", "lj"):
        if getattr(desc, key) is not None:
            out.append(key)
    return out


def run(path: str, precision=None, device: int = 0, steps=None, out=sys.stderr) -> dict:
    inp = load(path)
    d = inp.desc
    prec = precision or ("fp64" if inp.precision == "double" else "mixed")
    total = inp.total_step if steps is None else int(steps)
    save = max(1, inp.save_step)
    os.makedirs(inp.output_path, exist_ok=True)
    ene_path = os.path.join(inp.output_path, inp.output_prefix + ".ene")
    xyz_path = os.path.join(inp.output_path, inp.output_prefix + ".xyz")
    terms = _present(d)
    eng = Engine(prec, device=device)
    sid = eng.add_system(d)
    eng.commit()
    t0 = time.perf_counter()
    anneal = inp.schedule                    # SimulatedAnnealing: (first, last, each_step)
    r_total = 1.0 / total if total else 0.0
    with open(ene_path, "w") as ene, open(xyz_path, "w") as xyz:
        ene.write("# timestep " + " ".join(TERM_LABEL[t] for t in terms) + " kinetic_energy\n")
        done = 0
        while True:
            if done % save == 0 or done >= total:
                e = eng.energies(sid)
                p, v, _ = eng.state(sid)
                kin = 0.5 * float(np.sum(d.mass[:, None] * v * v))
                ene.write(f"{done} " + " ".join(f"{e[t]:.10e}" for t in terms) + f" {kin:.10e}\n")
                xyz.write(f"{d.n}\nstep = {done}\n")
                xyz.write("".join(f"X {x:.6f} {y:.6f} {z:.6f}\n" for x, y, z in p))
            if done >= total:
                break
            k = min(save - done % save, total - done)
            if anneal:
                k = min(k, anneal[2] - done % anneal[2])
            eng.step(k)
            done += k
            if anneal and done % anneal[2] == 0:    # core/SimulatedAnnealingSimulator.hpp:144-154
                eng.set_temperature(sid, current(anneal[0], anneal[1], done * r_total))
    wall = time.perf_counter() - t0
    eng.close()
    res = {"steps": total, "particles": d.n, "precision": prec, "wall_s": wall,
           "energy_file": ene_path, "trajectory": xyz_path}
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
