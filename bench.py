"""REMC benchmark: replica-steps/s and pair-energies/s on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload batch64]
                  [--impl ours|reference]

One bench step = one replica-exchange block of the workload: every replica of
every system advances `--block-steps` (default 1000) Metropolis steps in one
persistent sweep launch, followed by one exchange round, replayed as a CUDA
graph. `value` = replica-steps/s over the whole job (all ranks); inputs are
resident in HBM. `e2e` = the same metric through the C ABI with host buffers:
every step uploads the full replica state from host memory, runs one block and
reads state and energies back. Multi-GPU runs are weak scaling: each rank
advances its own independent batch (a different seed), with no collective on
the data path; the only collectives reduce the timings (max over ranks) and
the pair-evaluation counts (sum) after the timed region.

--impl reference times the reference's own CPU engine (Replica::MCSearch,
compiled from the reference sources into oracle/_ref) on bounded samples of
the same workload, with all host threads. The reference executable cannot
load more than 30 molecules (a double free in Replica::loadMolecule), so its
replicas are built and driven through the harness in oracle/_ref.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# algorithmic cost per pair evaluation (FMA = 2 FLOP): residue pair with
# Kim-Hummer contact + Debye-Hueckel = 41 FLOP + 2 MUFU (rsqrt, ex2);
# crowder pair = 26 FLOP + 1 MUFU (rsqrt). A dE pair is two evaluations.
FLOP_RESIDUE_PAIR = 41
FLOP_CROWDER_PAIR = 26
MUFU_RESIDUE_PAIR = 2
MUFU_CROWDER_PAIR = 1
FP32_LANES_PER_SM = 128


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="batch64",
                    choices=["batch64", "crowded", "two_chain", "assembly"])
    ap.add_argument("--block-steps", type=int, default=1000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--adjoint-snapshots", type=int, default=4096,
                    help="snapshots of the crowded system for the adjoint/energy cost ratio")
    ap.add_argument("--plain-steps", type=int, default=20,
                    help="MC steps of the per-replica-launch comparison sample")
    ap.add_argument("--schedule", default="",
                    help="THREADS,SMEM,CTAS: fixed sweep schedule instead of the autotuner")
    return ap.parse_args()


# ---------------------------------------------------------------- ranks
def rank_seed(seed: int, rank: int) -> int:
    """Workload seed of one rank: every rank generates its own batch."""
    return seed + 1000 * rank


def reduce_over_ranks(times, counts, world: int, device="cpu"):
    """Max over ranks of each per-rank time and sum of each per-rank count.
    Every rank calls this with lists of the same lengths at the same point,
    so all ranks issue the same two collectives in the same order."""
    if world == 1:
        return [float(x) for x in times], [float(x) for x in counts]
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x) for x in times], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if not counts:
        return t.tolist(), []
    c = torch.tensor([float(x) for x in counts], dtype=torch.float64, device=device)
    dist.all_reduce(c)
    return t.tolist(), c.tolist()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.proc = subprocess.Popen(
            ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
             "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            t = [x.strip() for x in ln.split(",")]
            if len(t) < 9:
                continue
            try:
                sm.append(float(t[1]))
                mx.append(float(t[2]))
            except ValueError:
                continue
            for nm, v in zip(names, t[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- reference CPU
PAIRS_PER_CORE_S = 2.5e7  # order of the reference E() rate per core (pairs/s)


def inter_molecular_pairs(system) -> int:
    """Pairs the reference's Replica::E() evaluates every MC step (all bead
    pairs of different molecules, Replica.cpp:603-745)."""
    n = system.n_beads
    return (n * (n - 1) - sum(m.n * (m.n - 1) for m in system.molecules)) // 2


def reference_sample_plan(workload, seed: int, cores: int, seconds: float):
    """Replicas of the workload for the reference engine and an MC step count
    so that one sample is about `seconds` of work on `cores` threads (the
    reference evaluates the full O(N^2) energy every step). Every system of
    the workload takes part with the same number of its replicas, so the
    sample has the workload's own mix of system sizes; a system's replicas
    differ only in temperature, and their cost per step is the same.
    Returns [(system index, ladder index)] and the MC step count."""
    n = len(workload.systems)
    per = max(1, min(min(workload.n_replicas), -(-2 * cores // n)))
    picks = []
    for si in range(n):
        R = workload.n_replicas[si]
        idx = sorted({int(round(k * (R - 1) / max(per - 1, 1))) for k in range(per)})
        picks.extend((si, k) for k in idx)
    pairs = sum(inter_molecular_pairs(workload.systems[si]) for si, _ in picks)
    mc = int(PAIRS_PER_CORE_S * cores * seconds / max(pairs, 1.0))
    return picks, max(2, min(mc, 2000))


def balanced_order(costs, threads: int):
    """Order of the replicas such that the contiguous slices the timing
    harness hands to its threads (main.cpp:879-883) carry near-equal work:
    each replica, in decreasing cost, joins the least loaded slice that still
    has room."""
    n = len(costs)
    threads = max(1, min(threads, n))
    per = -(-n // threads)
    slices = [[] for _ in range(threads)]
    load = [0.0] * threads
    for i in sorted(range(n), key=lambda i: -costs[i]):
        k = min((t for t in range(threads) if len(slices[t]) < per), key=lambda t: load[t])
        slices[k].append(i)
        load[k] += costs[i]
    return [i for sl in slices for i in sl]


def build_reference_replicas(workload, picks, threads: int = 1):
    """The reference's own Replica objects (oracle/_ref, compiled from its
    sources), one per (system, ladder index) pick, in an order that balances
    the harness's thread slices; the reference executable itself cannot load
    more than 30 molecules (double free in Replica::loadMolecule), so the
    replicas are built through the harness. Returns the replicas and their
    inter-molecular pair counts."""
    from oracle import bindings as ob
    costs = [inter_molecular_pairs(workload.systems[si]) for si, _ in picks]
    reps, pairs = [], []
    for i in balanced_order(costs, threads):
        si, k = picks[i]
        s = workload.systems[si]
        r = ob.ReferenceReplica(s, temperature=float(workload.ladders[si][k]))
        r.set_steps(workload.translate_step, workload.rotate_step)
        reps.append(r)
        pairs.append(costs[i])
    return reps, pairs


def maps_engine_library() -> bool:
    """True if this process has this repository's engine library mapped."""
    try:
        with open("/proc/self/maps") as fh:
            return "libremc_b200" in fh.read()
    except OSError:
        return False


def time_reference(reps, threads: int, mc: int):
    from oracle import bindings as ob
    return ob.time_reference_mcsearch(reps, threads, mc)


# ---------------------------------------------------------------- our arm
def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, world, rank)

    import numpy as np
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from remcdockingsimulator_b200 import synth
    from remcdockingsimulator_b200.engine import Engine

    w = synth.WORKLOADS[args.workload](rank_seed(args.seed, rank))
    eng = Engine(w.systems, w.n_replicas, w.params)
    eng.set_replica_params(w.ladders, np.full(len(w.systems), w.translate_step, np.float32),
                           np.full(len(w.systems), w.rotate_step))
    eng.energy_full()
    # the project's autotuner picks threads per replica, the shared-memory
    # layout and CTAs per replica for this batch (probe sweeps, state restored
    # afterwards), unless --schedule fixes them
    if args.schedule:
        t_, m_, c_ = (int(x) for x in args.schedule.split(","))
        eng.set_schedule(t_, bool(m_))
        eng.set_cluster(c_)
        sched_threads, sched_smem, chosen_by = t_, bool(m_), "--schedule"
    else:
        # probes as long as a timed block: the candidates differ by a few
        # percent, which shorter probes do not resolve reliably
        sched_threads, sched_smem, _ = eng.autotune(probe_steps=args.block_steps)
        chosen_by = "remc_autotune"
    stream = torch.cuda.ExternalStream(eng.stream_ptr(), device=torch.device("cuda", local))
    n_inst = eng.n_inst
    B = args.block_steps
    seed = 20241203 + rank

    # L2 flush buffer (> 126 MB L2), written between timed steps, outside the timing
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    step_ctr = 0
    for _ in range(args.warmup):
        eng.run(1, B, seed, step_ctr * B, step_ctr)
        step_ctr += 1
    eng.sync()
    eng.reset_counters()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            starts[k].record(stream)
        eng.run(1, B, seed, step_ctr * B, step_ctr)
        step_ctr += 1
        with torch.cuda.stream(stream):
            ends[k].record(stream)
            flush.fill_(float(k))
    eng.sync()
    barrier()
    clk = clocks.stop()
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    ev_res, ev_crowd = eng.pair_evaluations()
    timed_flop_step = (ev_res * FLOP_RESIDUE_PAIR + ev_crowd * FLOP_CROWDER_PAIR) / args.steps
    timed_mufu_step = (ev_res * MUFU_RESIDUE_PAIR + ev_crowd * MUFU_CROWDER_PAIR) / args.steps
    (t_max,), (pair_evals_all, inst_all) = reduce_over_ranks(
        [ms / 1000.0], [ev_res + ev_crowd, n_inst], world, "cuda")
    replica_steps = inst_all * B * args.steps
    value = replica_steps / t_max

    # ---- the dominant kernel (the persistent sweep) also timed alone, three
    # launches, as a cross-check of the per-step figure
    eng.reset_counters()
    rs, re_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n_roof = 3
    with torch.cuda.stream(stream):
        rs.record(stream)
    for k in range(n_roof):
        eng.sweep(B, seed + 1, (step_ctr + k) * B)
    with torch.cuda.stream(stream):
        re_.record(stream)
    eng.sync()
    sweep_ms = rs.elapsed_time(re_) / n_roof
    r_res, r_crowd = eng.pair_evaluations()
    flop_launch = (r_res * FLOP_RESIDUE_PAIR + r_crowd * FLOP_CROWDER_PAIR) / n_roof
    mufu_launch = (r_res * MUFU_RESIDUE_PAIR + r_crowd * MUFU_CROWDER_PAIR) / n_roof
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except OSError:
        pass
    sm_count = torch.cuda.get_device_properties(local).multi_processor_count
    max_mhz = float(peaks.get("sm_max_mhz") or clk.get("sm_max_mhz") or 1965.0)
    fp32_peak = sm_count * FP32_LANES_PER_SM * 2 * max_mhz * 1e6 / 1e12
    # achieved: the timed region's own sweeps (one launch per bench step),
    # algorithmic FLOP counted by the kernel over the time of the whole step
    # (which also holds the proposal, exchange and counter kernels, under 1 %)
    step_ms = ms / args.steps
    achieved = timed_flop_step / (step_ms / 1000.0) / 1e12
    roofline = {"bound": "fp32", "kernel": "sweep_kernel", "achieved": round(achieved, 3),
                "peak": round(fp32_peak, 2), "unit": "TFLOP/s", "frac": round(achieved / fp32_peak, 4),
                "peak_source": "nominal FP32 FMA issue rate (%d SMs x 128 lanes x 2) at the "
                               "measured max SM clock %.0f MHz (MEASURED_PEAKS.json has no FP32 "
                               "figure); the kernel is FP32/MUFU-bound, not HBM or tensor" %
                               (sm_count, max_mhz),
                "flop_per_launch": timed_flop_step, "launch_ms": round(step_ms, 4),
                "launch_ms_note": "CUDA events around each timed bench step (one sweep launch "
                                  "and its proposal, exchange and counter kernels)",
                "mufu_per_s": timed_mufu_step / (step_ms / 1000.0),
                "alone": {"launch_ms": round(sweep_ms, 4), "flop_per_launch": flop_launch,
                          "achieved": round(flop_launch / (sweep_ms / 1000.0) / 1e12, 3),
                          "note": "three further sweep launches timed on their own"},
                "traffic": None,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one sweep "
                                  "launch of this workload (profiles/traffic.json)"}
    prof_traffic = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(prof_traffic):
        try:
            with open(prof_traffic) as fh:
                roofline["traffic"] = json.load(fh).get(args.workload)
        except (OSError, ValueError):
            pass

    # ---- plain per-replica launches on a short sample (same trajectory rule)
    plain = None
    if args.plain_steps > 0:
        ps, pe = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            ps.record(stream)
        eng.sweep_plain(args.plain_steps, seed + 2, 0)
        with torch.cuda.stream(stream):
            pe.record(stream)
        eng.sync()
        (p_s,), _ = reduce_over_ranks([ps.elapsed_time(pe) / 1000.0], [], world, "cuda")
        p_ms = p_s * 1000.0
        plain_rate = inst_all * args.plain_steps / (p_ms / 1000.0)
        plain = {"value": plain_rate, "unit": "replica-steps/s", "steps": args.plain_steps,
                 "launches": n_inst * args.plain_steps,
                 "batched_over_plain": value / plain_rate}

    # ---- e2e through the C ABI with host buffers
    st = eng.download_state()
    host = [torch.from_numpy(a.copy()).pin_memory().numpy() for a in st]
    e2e_steps = max(2, min(args.steps, 5))
    barrier()
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        eng.upload_state(*host)              # pinned host -> device, checked and packed on the GPU
        eng.run(1, B, seed + 3, k * B, k)
        eng.download_state(out=host)         # device -> the same pinned buffers
        en = eng.energies()
    eng.sync()
    (t_e2e,), _ = reduce_over_ranks([time.perf_counter() - t0], [], world, "cuda")
    h2d = sum(a.nbytes for a in host)
    d2h = h2d + en.nbytes
    e2e = {"value": inst_all * B * e2e_steps / t_e2e, "unit": "replica-steps/s",
           "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
           "path": "remc_upload_state + remc_run + remc_download_state + remc_get_energies"}

    # ---- adjoint cost against one energy evaluation: 4096 snapshots of the
    # crowded system (all replicas of one system, decorrelated by a sweep)
    adjoint = None
    if args.adjoint_snapshots > 0:
        wa = synth.crowded(rank_seed(args.seed + 7, rank))
        ea = Engine(wa.systems, [args.adjoint_snapshots], wa.params)
        ea.set_replica_params([np.linspace(290, 480, args.adjoint_snapshots).astype(np.float32)],
                              [wa.translate_step], [wa.rotate_step])
        ea.energy_full()
        ea.sweep(200, seed + 9, 0)
        ea.sync()
        sa = torch.cuda.ExternalStream(ea.stream_ptr(), device=torch.device("cuda", local))
        times = {}
        for name, fn in (("energy", lambda: ea.energy_full_async()),
                         ("adjoint", lambda: ea.adjoint_kernels())):
            fn()
            ea.sync()
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(sa):
                a0.record(sa)
            for _ in range(5):
                fn()
            with torch.cuda.stream(sa):
                a1.record(sa)
            ea.sync()
            times[name] = a0.elapsed_time(a1) / 5
        adjoint = {"snapshots": args.adjoint_snapshots, "energy_ms": times["energy"],
                   "adjoint_ms": times["adjoint"],
                   "adjoint_over_energy": times["adjoint"] / times["energy"],
                   "outputs": "per-bead forces, per-molecule force+torque, dE/dlambda, "
                              "dE/dXi, dE/deps[20x20]"}
        ea.close()

    # ---- CPU baseline (reference engine, bounded sample), rank 0 at N = 1
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(w, args.seed)

    # per timed step: ctrl_set_kernel (remc_run) + the graph's proposal_kernel,
    # block_cost_kernel and rank_kernel (work order by proposal cost, single
    # CTAs per replica), sweep_kernel, exchange_kernel and ctrl_advance_kernel
    gpu_launches = args.steps * (3 + eng.work_order()[1])
    if rank == 0:
        line = {
            "metric": "REMC replica-steps/s (batched persistent sweep + CUDA graph)",
            "value": value, "unit": "replica-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max * 1000.0 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
            "data": "synthetic (seeded generator with the benchmark configuration's shapes)",
            "config": {"workload": w.name, "description": w.description,
                       "systems": len(w.systems), "replica_instances": n_inst,
                       "beads_per_replica_mean": sum(s.n_beads * r for s, r in
                                                     zip(w.systems, w.n_replicas)) / n_inst,
                       "mc_steps_per_bench_step": B, "exchange_every": B,
                       "l2": "256 MB buffer written between timed steps, outside the timing",
                       "schedule": {"threads_per_replica": sched_threads,
                                    "molecule_data_in_shared_memory": sched_smem,
                                    "ctas_per_replica": eng.schedule()[2],
                                    "chosen_by": chosen_by},
                       "parallelism": "replicas" if world == 1 else "weak: %d independent batches" % world},
            "pair_energies_per_s": pair_evals_all / t_max,
            "pair_energy_note": "pair evaluations per second; a dE pair counts twice",
            "roofline": roofline, "plain": plain, "e2e": e2e, "cpu_baseline": cpu,
            "adjoint": adjoint,
            "clocks": clk, "gpu_launches": gpu_launches,
        }
        print(json.dumps(line))
    eng.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def cpu_baseline(workload, seed: int):
    cores = os.cpu_count() or 1
    try:
        picks, mc = reference_sample_plan(workload, seed, cores, 10.0)
        threads = min(cores, len(picks))
        reps, pairs = build_reference_replicas(workload, picks, threads)
        wall = time_reference(reps, threads, mc)
        n_rs = len(reps) * mc
        # the reference's own Replica::E() on one core (its "Host Timer" figure,
        # Replica.cpp:1082): inter-molecular pairs evaluated per second
        r0 = reps[0]
        calls, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < 1.0:
            r0.E()
            calls += 1
        e_rate = pairs[0] * calls / (time.perf_counter() - t0)
        for r in reps:
            r.close()
        n_sys = len({si for si, _ in picks})
        return {"value": n_rs / wall, "unit": "replica-steps/s", "cores": threads,
                "pair_energies_per_s": sum(pairs) * mc / wall,
                "e_pairs_per_s_one_core": e_rate,
                "kind": "reference",
                "sample": "reference Replica::MCSearch (compiled from its sources, full energy "
                          "every step, its own (6/r)^6 crowder model and lambda=0.159) on %d "
                          "replicas (%d of each of the %d of %d systems) x %d MC steps, %d "
                          "threads, %.1f s" %
                          (len(reps), len(reps) // max(n_sys, 1), n_sys,
                           len(workload.systems), mc, threads, wall)}
    except Exception as exc:  # reported, not fatal: the GPU number stands alone
        return {"value": None, "unit": "replica-steps/s", "cores": 0, "kind": "reference",
                "sample": "failed: %s" % str(exc)[:300]}


def reference_arm(args, world: int, rank: int):
    if rank != 0:
        return 0
    from oracle import bindings as ob
    if not ob.reference_available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference CPU engine not built in oracle/_ref"}))
        return 0
    from remcdockingsimulator_b200 import synth
    w = synth.WORKLOADS[args.workload](args.seed)
    cores = os.cpu_count() or 1
    picks, mc = reference_sample_plan(w, args.seed, cores, 4.0)
    threads = min(cores, len(picks))
    reps, pairs = build_reference_replicas(w, picks, threads)
    for _ in range(args.warmup):
        time_reference(reps, threads, max(1, mc // 8))
    total_t = 0.0
    for _ in range(args.steps):
        total_t += time_reference(reps, threads, mc)
    for r in reps:
        r.close()
    value = len(reps) * mc * args.steps / total_t
    pair_rate = sum(pairs) * mc * args.steps / total_t
    n_sys = len({si for si, _ in picks})
    sample = ("reference Replica::MCSearch (compiled from its sources, full energy every step, "
              "its own (6/r)^6 crowder model and lambda=0.159) on %d replicas (%d of each of "
              "the %d of %d systems, so the batch's own mix of sizes) x %d MC steps per bench "
              "step, %d threads" % (len(reps), len(reps) // max(n_sys, 1), n_sys, len(w.systems),
                                    mc, threads))
    line = {
        "impl": "reference",
        "metric": "REMC replica-steps/s (batched persistent sweep + CUDA graph)",
        "value": value, "unit": "replica-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_t * 1000.0 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
        "data": "synthetic (seeded generator with the benchmark configuration's shapes)",
        "config": {"workload": w.name, "description": w.description,
                   "sample_replicas": len(reps), "sample_systems": n_sys,
                   "mc_steps_per_sample": mc},
        "pair_energies_per_s": pair_rate,
        "pair_energy_note": "pairs of the full energy the reference evaluates every MC step",
        "engine_library_mapped": maps_engine_library(),
        "cpu_baseline": {"value": value, "unit": "replica-steps/s", "cores": threads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "replica-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
