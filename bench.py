"""Benchmark of the B200 Mjolnir hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Workload (the batching configuration the headline metric is quoted on): 256
independent coarse-grained polymer melts, sizes log-uniform in [500, 20000]
beads (chains of ~200 beads, 10,000 beads per 300 A sphere density), per-system
temperature U[280, 360] K and ionic strength U[0.05, 0.3] M; harmonic bonds and
angles, cosine dihedrals, ExcludedVolume and DebyeHuckel with cell lists
(margin 0.5), BAOAB at dt = 0.01.  All systems are packed into one arena and
advanced by the same CUDA-graph step.  Synthetic, seeded inputs: there is no
dataset.

One bench step = CHUNK (100) MD steps of every system.  `value` is aggregate
particle-steps/s with the state resident in HBM, timed with CUDA events on the
library's stream; `e2e` is the same metric through the public C ABI with the
positions and velocities uploaded from pinned host memory before and
downloaded after every bench step.  Under torchrun every rank runs its own
replica of the batch (replicas only: no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CHUNK = 100
NSYS = 256
SEED = 4


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nsys", type=int, default=NSYS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--serve", type=float, default=20.0,
                    help="seconds of the Poisson serving run; 0 skips it")
    ap.add_argument("--no-fluid", action="store_true",
                    help="skip the pair-kernel roofline on the 1,048,576-bead periodic fluid")
    ap.add_argument("--no-precision", action="store_true",
                    help="skip the 2,000-step precision report on the 1,048,576-bead fluid")
    ap.add_argument("--no-fluid-reference", action="store_true",
                    help="skip timing the reference's OpenMP path on the 1,048,576-bead fluid (about a minute)")
    return ap.parse_args()


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return ws, rank, local, pg


def max_over_ranks(x, pg):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []
        self.span = [0, None]          # lines that arrived between mark_start and mark_end

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first(self, seconds=3.0):
        """Until the first sample arrives (nvidia-smi takes a moment to start)."""
        t0 = time.time()
        while self.proc and not self.lines and time.time() - t0 < seconds:
            time.sleep(0.02)

    def mark_start(self):
        self.span[0] = len(self.lines)

    def mark_end(self):
        # the sample in flight when the region ends still saw it
        time.sleep(0.11)
        self.span[1] = len(self.lines)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.lines[self.span[0]:self.span[1]] or self.lines[self.span[0]:] or self.lines
        for ln in lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def ncu_traffic(key, schedule, slots, half=False):
    """(DRAM bytes of one launch, source text) from profiles/ncu_traffic.json
    for the kernel `key` captured with the same schedule and list form, scaled
    by slots; (None, reason) when no capture of that kernel, schedule and list
    form is recorded."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            rec = json.load(f)[key]
    except Exception:
        return None, "no ncu capture recorded for this kernel"
    if rec.get("schedule") != schedule:
        return None, f"the recorded capture is of schedule {rec.get('schedule')}, this launch runs {schedule}"
    if bool(rec.get("half_lists", False)) != bool(half):
        form = lambda h: "half" if h else "full"
        return None, (f"the recorded capture walks {form(rec.get('half_lists', False))} lists, "
                      f"this launch {form(half)} lists")
    b = (rec["dram_read_bytes"] + rec["dram_write_bytes"]) / rec["slots"] * slots
    return b, (f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch ({rec['kernel']}, "
               f"{rec['slots']} slots, {rec['workload']}), scaled by slots; profiles/ncu_traffic.json")


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def build_batch(nsys, synth=None):
    from mjolnir_b200 import systems as S
    return S.polymer_batch(nsys=nsys, seed=SEED, synth=synth)


# ---------------------------------------------------------------- reference
class ReferenceBatch:
    """The reference's own OpenMP path (oracle/_ref: OpenMPSimulatorTraits,
    BAOAB, cell lists, the unmodified reference headers) holding every system
    of a batch, stepped one system after another as the reference would run
    separate simulations.  Both the reference arm and the cpu_baseline leg
    time the batch through this class, so the two agree by construction."""

    def __init__(self, descs):
        import oracle
        self.descs = descs
        self.n = sum(d.n for d in descs)
        self.sims = []
        for d in descs:
            r = oracle.Reference(d, parallel=True)
            r.initialize()
            self.sims.append(r)
        self.threads = oracle.Reference.max_threads()

    def run(self, md_steps, part=0, parts=1):
        """Advances the systems k with k % parts == part (every system by
        default) by md_steps; returns (seconds spent in the reference's
        integrator steps, particle-steps done); input and initialisation are
        excluded."""
        t, ps = 0.0, 0
        for k, (r, d) in enumerate(zip(self.sims, self.descs)):
            if k % parts == part:
                t += r.run(md_steps)
                ps += d.n * md_steps
        return t, ps

    def close(self):
        for r in self.sims:
            r.close()


def omp_setup():
    """OpenMP placement of the reference's threads: every host thread, bound
    close (set before the reference library starts its runtime)."""
    os.environ.setdefault("OMP_PROC_BIND", "close")
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    return {"omp_num_threads": os.environ["OMP_NUM_THREADS"], "omp_proc_bind": os.environ["OMP_PROC_BIND"]}


def reference_descs(nsys):
    """The benchmark batch built with the seeded builders as compiled into
    the reference driver (oracle/_ref), so the reference arm never loads the
    product library; the same source makes the same systems."""
    import oracle
    return build_batch(nsys, synth=oracle.synthetic_library())


def cpu_reference_rate(descs, budget_s=12.0):
    """cpu_baseline leg: a bounded sample of the timed workload on the
    reference's OpenMP path -- every system of the batch, CHUNK-step rounds
    until `budget_s` of integrator time; returns (particle-steps/s, sample
    text, threads)."""
    import oracle
    if not oracle.reference_available():
        return None
    rb = ReferenceBatch(descs)
    t, ps, steps = 0.0, 0, 0
    md = max(1, CHUNK // 10)
    while t < budget_s:
        dt, dps = rb.run(md)
        t += dt
        ps += dps
        steps += md
    rb.close()
    sample = (f"all {len(descs)} systems ({rb.n} beads), {steps} MD steps each, one system after another "
              f"through OpenMPSimulatorTraits BAOAB ({rb.threads} threads)")
    return ps / t, sample, rb.threads


def fluid_reference(steps=20, margins=(0.2, 0.2)):
    """The reference's OpenMP path on the 1,048,576-bead fluid (the
    precision-at-scale configuration, at the precision report's margins), a
    bounded sample: building the reference's objects (which makes its
    exclusion and cell lists once) is timed apart, then `steps` MD steps,
    which include the list rebuilds its margin logic triggers."""
    import time
    import oracle
    from mjolnir_b200 import systems as S
    if not oracle.reference_available():
        return None
    omp = omp_setup()
    d = S.bead_fluid(n=1 << 20, density=0.003, seed=3, synth=oracle.synthetic_library())
    d.exv.margin, d.dh.margin = margins
    t0 = time.perf_counter()
    r = oracle.Reference(d, parallel=True)
    r.initialize()
    t_build = time.perf_counter() - t0
    t_steps = r.run(steps)
    r.close()
    return {"value": d.n * steps / t_steps, "unit": "particle-steps/s", "kind": "reference",
            "cores": oracle.Reference.max_threads(), **omp, "beads": d.n, "steps_timed": steps,
            "s_per_step": t_steps / steps, "setup_s": t_build,
            "sample": f"{steps} MD steps of the 1,048,576-bead fluid (margins {margins[0]} / {margins[1]}) "
                      "through OpenMPSimulatorTraits BAOAB, list rebuilds included; setup timed apart"}


# the reference arm's bench step: CHUNK MD steps of every REF_PARTS-th system,
# the subset rotating from step to step, so that a run of the driver's length
# (tens of bench steps) ends within a few minutes on the host's cores
REF_PARTS = 2


def run_reference_arm(args, ws, rank, pg):
    """--impl reference: the reference's own CPU implementation on the same
    workload and config as the B200 arm; one bench step = CHUNK MD steps of
    half the systems of the batch (alternate halves from step to step, a
    bounded sample).  Under torchrun only rank 0 runs it."""
    if rank != 0:
        return
    import oracle
    omp = omp_setup()
    if not oracle.reference_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference driver oracle/_ref was not built (reference tree absent at build time)"}))
        return
    descs = reference_descs(args.nsys)
    rb = ReferenceBatch(descs)
    for k in range(args.warmup):
        rb.run(CHUNK, k % REF_PARTS, REF_PARTS)
    t, ps = 0.0, 0
    for k in range(args.steps):
        dt, dps = rb.run(CHUNK, k % REF_PARTS, REF_PARTS)
        t += dt
        ps += dps
    value = ps / t
    line = {
        "metric": "particle-steps/s (batched polymer systems)", "value": value, "unit": "particle-steps/s",
        "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(descs),
        "precision": "fp64 (the reference's OpenMP CPU path)",
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": rb.threads, "kind": "reference",
                         "sample": f"each bench step: {CHUNK} MD steps of every {REF_PARTS}nd of the "
                                   f"{len(descs)} systems (the halves alternating), one system after another "
                                   f"through OpenMPSimulatorTraits", **omp},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    rb.close()
    print(json.dumps(line))


def pair_kernels(eng, descs, sys_id, precision, label="batch"):
    """Time and algorithmic bytes of each pair kernel launch (slot gather +
    pair kernel).  Algorithmic bytes per launch: per participant its position
    and parameter (16 B as float4 in the mixed form, 32 B as double4 in FP64)
    and its force written (3 x 8 B), plus one 4-byte index per non-excluded
    pair inside the cutoff (P_cut, margin-free)."""
    out = {}
    per_slot = (16 if precision == "mixed" else 32) + 24
    import torch
    for term in ("exv", "dh"):
        torch.cuda.nvtx.range_push(f"{label}_{precision}_{term}")   # profiler selection
        ms = eng.time_kernel(term, reps=20)
        torch.cuda.nvtx.range_pop()
        pcut = eng.pair_count(sys_id, term)
        nslots = sum(len(getattr(d, term).idx) for d in descs)
        bytes_alg = nslots * per_slot + 4 * pcut
        out[term] = {"ms": ms, "pcut": pcut, "slots": nslots, "bytes": bytes_alg,
                     "gbs": bytes_alg / (ms * 1e-3) / 1e9}
    return out


def fluid_pair_roofline(local, peak, steps=200):
    """The precision-at-scale fluid as one plain system: 1,048,576 beads at
    0.003 per cubic A in a periodic cube, ExcludedVolume on all beads and
    DebyeHuckel on 30 % (I = 0.15 M, T = 300 K, BAOAB dt = 0.3).  Per form:
    margins and launch shapes autotuned on whole steps, then the whole-step
    rate (particle-steps/s over `steps` MD steps) and the pair kernels."""
    import torch
    from mjolnir_b200 import autotune
    from mjolnir_b200 import systems as S
    from mjolnir_b200.engine import Engine
    d = S.bead_fluid(n=1 << 20, density=0.003, seed=3)
    out = {"beads": d.n}
    for prec in ("fp64", "mixed"):
        e = Engine(prec, device=local)
        e.add_system(d)
        e.commit()
        e.step(2)
        tuned = autotune.tune(e, terms=("exv", "dh"), margins=(0.05, 0.1, 0.2, 0.3), steps=100, warm=100)
        stream = torch.cuda.ExternalStream(e.stream_handle(), device=local)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        e.step(20)
        a.record(stream)
        e.step(steps)
        b.record(stream)
        b.synchronize()
        step_ms = a.elapsed_time(b) / steps
        k = pair_kernels(e, [d], 0, prec, label="fluid")
        for term, v in k.items():
            v["traffic"], v["traffic_source"] = ncu_traffic(f"fluid1m_{term}" if prec == "mixed" else "",
                                                            e.get_pair_schedule(term), v["slots"],
                                                            prec == "mixed" and e.get_half_lists(term))
        tot_b = sum(v["bytes"] for v in k.values())
        tot_ms = sum(v["ms"] for v in k.values())
        out[prec] = {"terms": k, "tuned": tuned, "gbs": tot_b / (tot_ms * 1e-3) / 1e9,
                     "frac": tot_b / (tot_ms * 1e-3) / 1e9 / peak, "ms": tot_ms,
                     "ms_per_md_step": step_ms, "particle_steps_per_s": d.n / (step_ms * 1e-3)}
        e.close()
    return out


def small_configs(local, steps=2000, cpu_budget_s=3.0):
    """The two single-system configurations: the 4,096-particle Lennard-Jones
    fluid (reduced density 0.8, cutoff 2.5, BAOAB dt 0.005) and the
    10,000-bead polymer melt in unbounded space (50 chains x 200 beads), each
    as one plain system on the GPU in both forms (`steps` MD steps after a
    warm-up, CUDA events on the library's stream), beside the reference's own
    OpenMP path stepping the same system (a bounded sample)."""
    import torch
    from mjolnir_b200 import systems as S
    from mjolnir_b200.engine import Engine
    out = {}
    for name, d in (("lj_fluid_4096", S.lj_fluid(n=4096, density=0.8, margin=0.2, seed=1)),
                    ("polymer_melt_10000", S.polymer_melt(nchains=50, nbeads=200, radius=300.0, seed=2))):
        row = {"particles": d.n}
        for prec in ("fp64", "mixed"):
            e = Engine(prec, device=local)
            e.add_system(d)
            e.commit()
            e.step(200)
            e.synchronize()
            st = torch.cuda.ExternalStream(e.stream_handle(), device=local)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(st)
            e.step(steps)
            b.record(st)
            b.synchronize()
            row[prec] = d.n * steps / (a.elapsed_time(b) / 1e3)
            e.close()
        res = cpu_reference_rate([d], budget_s=cpu_budget_s) if cpu_budget_s > 0 else None
        if res:
            row["reference_cpu"] = {"value": res[0], "cores": res[2], "kind": "reference"}
            row["fp64_over_reference"] = row["fp64"] / res[0]
        out[name] = row
    out["unit"] = "particle-steps/s"
    return out


def force_error(eng, descs, sids, local, nsample=16):
    """Per term, the largest relative RMS force error (sqrt(sum |dF|^2 /
    sum |F|^2)) of the mixed-form engine against the FP64 form evaluated on
    the mixed engine's own current coordinates, over `nsample` systems spread
    across the batch's sizes.  The FP64 form matches the reference's
    arithmetic (lists bit-exact, forces within 1e-12), so it stands in for the
    reference on coordinates the CPU never reaches."""
    from mjolnir_b200.engine import Engine
    order = sorted(range(len(descs)), key=lambda k: descs[k].n)
    pick = sorted({order[int(round(q * (len(order) - 1) / max(1, nsample - 1)))] for q in range(nsample)})
    fp = Engine("fp64", device=local)
    fsids = [fp.add_system(descs[k]) for k in pick]
    fp.commit()
    terms = ("bond", "angle", "dihedral", "exv", "dh")
    worst = {t: 0.0 for t in terms}
    for k, fs in zip(pick, fsids):
        pos, vel, _ = eng.state(sids[k])
        fp.set_state(fs, pos, vel)
        for t in terms:
            fm, _ = eng.term_force(sids[k], t)
            fd, _ = fp.term_force(fs, t)
            den = float(np.sum(fd * fd))
            err = float(np.sqrt(np.sum((fm - fd) ** 2) / den)) if den > 0 else 0.0
            worst[t] = max(worst[t], err)
    fp.close()
    return {"max_rel_rms": worst, "bound": 1e-5, "systems": len(pick),
            "reference": "FP64 form on the mixed trajectory's coordinates after the timed steps"}


def workload_config(descs):
    """The workload both arms run (identical dicts in both JSON lines)."""
    return {
        "workload": "batch of 256 independent polymer melts (bonds, angles, dihedrals, "
                    "ExcludedVolume, DebyeHuckel), log-uniform 500-20000 beads, "
                    "T U[280,360] K, I U[0.05,0.3] M",
        "systems": len(descs), "particles": int(sum(d.n for d in descs)),
        "md_steps_per_bench_step": CHUNK,
        "integrator": "BAOAB dt=0.01 gamma=1",
        "partition": "cell lists (PeriodicGridCellList / UnlimitedGridCellList), relative margin per term",
        "l2": "inputs larger than L2 (resident arena of several hundred MB)",
    }


# ---------------------------------------------------------------- B200 arm
def run_b200(args, ws, rank, local, pg):
    import torch
    torch.cuda.set_device(local)
    from mjolnir_b200.engine import Engine

    descs = build_batch(args.nsys)
    ntot = sum(d.n for d in descs)
    eng = Engine("mixed", device=local)
    sids = [eng.add_system(d) for d in descs]
    eng.commit()
    stream = torch.cuda.ExternalStream(eng.stream_handle(), device=local)
    tuned = None
    if not args.no_tune:
        from mjolnir_b200 import autotune
        tuned = autotune.tune(eng, log=lambda m: print(m, file=sys.stderr))

    # ---- device-resident throughput (the clock samples kept are those taken
    # during the timed steps; the sampler starts before the warm-up)
    with ClockSampler(local) as clocks:
        clocks.wait_first()
        for _ in range(args.warmup):
            eng.step(CHUNK)
        eng.synchronize()
        barrier(pg)
        l0 = eng.launch_count()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        clocks.mark_start()
        torch.cuda.nvtx.range_push("timed")     # profilers select the timed launches by this range
        e0.record(stream)
        for _ in range(args.steps):
            eng.step(CHUNK)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        clocks.mark_end()
    launches = eng.launch_count() - l0
    t_dev = e0.elapsed_time(e1) / 1e3
    t_dev = max_over_ranks(t_dev, pg)
    barrier(pg)
    value = ws * ntot * CHUNK * args.steps / t_dev

    # ---- end to end through the C ABI with pinned host buffers
    pos = torch.empty((ntot, 3), dtype=torch.float64, pin_memory=True).numpy()
    vel = torch.empty((ntot, 3), dtype=torch.float64, pin_memory=True).numpy()
    eng.get_state_all(pos, vel)
    e2e_steps = max(2, args.steps // 2)
    eng.set_state_all(pos, vel)
    eng.step(CHUNK)
    eng.get_state_all(pos, vel)
    barrier(pg)
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(e2e_steps):
        eng.set_state_all(pos, vel)        # H2D of the step's inputs
        eng.step(CHUNK)
        eng.get_state_all(pos, vel)        # D2H of the step's result
    f1.record(stream)
    f1.synchronize()
    t_e2e = max_over_ranks(f0.elapsed_time(f1) / 1e3, pg)
    e2e = ws * ntot * CHUNK * e2e_steps / t_e2e
    h2d = 2 * pos.nbytes
    d2h = 2 * pos.nbytes

    # ---- roofline of the dominant kernel (the pair kernels)
    peak, peak_kind = measured_peaks()
    kern = pair_kernels(eng, descs, -1, "mixed")
    dom = max(kern, key=lambda k: kern[k]["ms"])
    k = kern[dom]
    # DRAM bytes (read + write) of one launch of this kernel as ncu measured
    # them (profiles/ncu_traffic.json: per kernel and workload, the capture's
    # bytes and slots), scaled to this launch by its slots
    traffic, traffic_src = ncu_traffic(f"batch256_{dom}", eng.get_pair_schedule(dom), k["slots"],
                                       eng.get_half_lists(dom))
    local_ms = {t: eng.time_kernel(t, reps=20) for t in ("bond", "angle", "dihedral")}
    shape = eng.get_pair_schedule(dom), eng.get_threads_per_particle(dom), eng.get_pair_unroll(dom)
    roofline = {"bound": "hbm", "kernel": f"pair force kernel of {dom} (schedule {shape[0]}, "
                f"{shape[1]} threads or words per slot, {shape[2]} partners per batch, "
                f"{'half' if eng.get_half_lists(dom) else 'full'} lists)",
                "achieved": k["gbs"], "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                "frac": k["gbs"] / peak, "traffic": traffic,
                "traffic_source": traffic_src,
                "timing": "CUDA events per launch on the library stream, L2 evicted before each launch",
                "ms_per_launch": k["ms"], "pairs_in_cutoff": k["pcut"],
                "algorithmic_bytes": k["bytes"], "other": {t: kern[t] for t in kern if t != dom},
                "local_ms_per_launch": local_ms}

    # ---- plain single-system FP64 path: every system of the batch, one at a time
    plain = None
    if not args.no_plain and rank == 0:
        tot_ps, tot_t = 0, 0.0
        pe = Engine("fp64", device=local)
        ps = torch.cuda.ExternalStream(pe.stream_handle(), device=local)
        for d in descs:
            sid = pe.add_system(d)
            pe.commit()
            pe.step(5)
            pe.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(ps)
            pe.step(CHUNK)
            b.record(ps)
            b.synchronize()
            tot_t += a.elapsed_time(b) / 1e3
            tot_ps += d.n * CHUNK
            pe.remove_system(sid)
        pe.close()
        plain = {"value": tot_ps / tot_t, "unit": "particle-steps/s",
                 "sample": f"all {len(descs)} systems run one at a time (one system per arena), FP64, "
                           f"{CHUNK} MD steps each, CUDA events per system",
                 "batched_over_plain": value / ws / (tot_ps / tot_t)}

    # ---- force error of the timed mixed-form run against the FP64 form
    ferr = force_error(eng, descs, sids, local) if rank == 0 else None

    # ---- the single-system configurations (LJ fluid, 10k-bead melt), GPU and reference CPU
    small = None
    if not args.no_plain and rank == 0 and ws == 1:
        small = small_configs(local, cpu_budget_s=0.0 if args.no_cpu_baseline else 3.0)

    # ---- pair kernels on the 1,048,576-bead periodic fluid, plain FP64 and mixed
    fluid = None
    if not args.no_fluid and rank == 0:
        fluid = fluid_pair_roofline(local, peak)

    # ---- precision at scale: the fluid's mixed trajectory against the FP64 form
    prec = None
    if not args.no_precision and rank == 0:
        from mjolnir_b200 import precision
        res = precision.run(steps=2000, every=1000, device=local)
        prec = {k: res[k] for k in ("beads", "steps", "every", "margin", "worst_force_rel_rms",
                                    "worst_total_force_rel_rms", "worst_energy_rel", "rebuilds")}
        prec["frames"] = [{"step": f["step"], **{t: f[t]["force_rel_rms"] for t in ("exv", "dh")},
                           "total": f["total_force_rel_rms"]} for f in res["frames"]]
        prec["bound"] = 1e-5
        prec["note"] = ("forces: mixed form vs the FP64 form on the mixed trajectory's coordinates every "
                        "1,000 steps; energies are evaluated in FP64 in both forms")

    # ---- the reference's OpenMP path on the 1 M fluid, a bounded sample
    if not args.no_fluid_reference and not args.no_cpu_baseline and rank == 0 and ws == 1:
        fref = fluid_reference()
        if fluid is not None and fref is not None:
            fluid["reference_cpu"] = fref
            fluid["mixed_over_reference"] = fluid["mixed"]["particle_steps_per_s"] / fref["value"]

    # ---- serving: Poisson arrivals at 200 jobs/s, continuous batching
    serving = None
    if args.serve > 0 and rank == 0 and ws == 1:
        from mjolnir_b200.serve import serve_poisson
        serving = serve_poisson(duration=args.serve, rate=200.0, tuned=tuned)
        serving["tuned"] = tuned is not None
        serving["note"] = ("offered load far above one GPU: most arrivals stay queued; "
                           "latency is over completed jobs")

    # ---- CPU baseline: the reference's OpenMP path on a bounded sample
    cpu = None
    if not args.no_cpu_baseline and rank == 0 and ws == 1:
        try:
            omp = omp_setup()
            res = cpu_reference_rate(descs, budget_s=12.0)
            if res:
                rate, sample, threads = res
                cpu = {"value": rate, "unit": "particle-steps/s", "cores": threads, "kind": "reference",
                       "sample": sample, **omp}
        except Exception as ex:  # the baseline must not sink the GPU line
            cpu = {"value": None, "error": str(ex)[:200]}

    if rank == 0:
        line = {
            "metric": "particle-steps/s (batched polymer systems)", "value": value, "unit": "particle-steps/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_dev / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 pair math, f64 state, i64 fixed-point forces",
            "data": "synthetic",
            "config": workload_config(descs),
            "precision": "mixed: FP32 pair and bonded math from FP64 displacements, int64 fixed-point "
                         "force sums, FP64 state and integrator",
            "autotuned": tuned,
            "e2e": {"value": e2e, "unit": "particle-steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "plain_fp64_single_system": plain,
            "single_system_configs": small,
            "force_error": ferr,
            "fluid_1m_pair_kernels": fluid,
            "precision_fluid_1m": prec,
            "serving": serving,
        }
        print(json.dumps(line))
    eng.close()


def main():
    args = parse()
    ws, rank, local, pg = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference_arm(args, ws, rank, pg)
        else:
            run_b200(args, ws, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
