"""Benchmark: events/sec of the B200 Independent-algorithm backend.

Workload (default): the batched sweep of 256 SpatiallyImplicit simulations
(local community J = floor(10^U(3,6)) cells of deme 1, metacommunity 1e7
cells, migration U(0.01, 0.2), speciation 10^U(-6,-3), seeds 0..255) run
to completion in one batched launch per round.  One step = one full batch.

  value      events/sec of the learned-scheduled kernel (the step queue
             ordered by the lifetime model, trained first on traces the
             backend generates, and the model's longest-lived simulations in
             engines of their own) with the origins resident in HBM (device
             time of the whole batch measured with CUDA events by the
             library, max over ranks), events = executed lineage steps;
             simulations down to 8 lineages continue in the per-simulation
             resident kernel on a stream of their own (both arms)
  plain      the same for the plain (unordered) kernel on the same workload,
             with `learned_over_plain` and `outcomes_identical` (the two arms'
             steps, species, speciation and duplicate counts, times)
  e2e        the same metric through the public C ABI call
             necsim_gpu_simulate_batch with host buffers: scenario set-up,
             host->device origin upload, simulation, device->host events;
             `parts` times a resident batch's set-up, run and release once
  timeline   when the last priority and other simulations ended, on the
             device clock from the batch's first round
  roofline   the round kernels (cooperative + step kernel) against their
             integer-issue bound: algorithmic wymum work per event on the
             canonical schedule (counted by the oracle) x events / kernel
             time, over the measured hash-issue peak; hbm_roofline gives
             their algorithmic bytes against the measured HBM bandwidth
  cpu_baseline  the CPU restatement of the reference's Independent
             algorithm on a bounded sample of the same workload (all
             simulations to t = 400), with the host CPU model
  same_slice the GPU's rate on exactly that sample (like for like with the
             CPU baseline and the reference arm)
  secondary  C3 in full and C5 to t = 400: the plain kernel's device rate
             beside the CPU restatement on the same horizon

`--impl reference` times that CPU restatement alone (all host cores) and
prints its line.  Multi-GPU (`--gpus N` under torchrun) runs N independent
replicas of the batch (weak scaling, no data-path collective).
"""
import argparse
import concurrent.futures
import importlib
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "events/sec on 1 B200: learned-scheduled vs plain independent kernel, bit-exact"
UNIT = "events/s"
L2_BYTES = 126 * 1024 * 1024


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="c4", choices=["c4", "c4-small", "c5", "c2", "c3", "c1"])
    p.add_argument("--schedule", default="both", choices=["plain", "learned", "both"],
                   help="both: time the plain and the learned-scheduled kernel on the same workload "
                        "(the line's value is the learned arm's)")
    p.add_argument("--autotune", default="auto", choices=["auto", "on", "off"],
                   help="pick block size, step_slice and dedup factor by timing a paused sample first "
                        "(auto: on for the batched sweeps)")
    p.add_argument("--train-pause", type=float, default=None,
                   help="pause_before of the trace runs that train the lifetime model (default: to "
                        "completion, so that every snapshotted lineage has its remaining events as label)")
    p.add_argument("--cpu-sample-pause", type=float, default=400.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--once", action="store_true",
                   help="profiling aid: one run of the workload's batch (plain schedule, the resident "
                        "kernel as in the timed arm), then print its events and device time; no timing "
                        "arms, baselines or training")
    p.add_argument("--no-secondary", action="store_true",
                   help="skip the secondary workloads (C3 in full, C5 to t=400) beside the sweep")
    p.add_argument("--pause", type=float, default=None,
                   help="pause_before of every simulation (default: run to completion)")
    p.add_argument("--event-time-sampler", default="poisson", choices=["poisson", "exp"],
                   help="poisson: the Independent algorithm's PoissonEventTimeSampler (the headline); "
                        "exp: the CUDA algorithm's ExpEventTimeSampler, -ln(U(0,1]) / lambda per event")
    return p.parse_args()


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
def workload(name):
    """(description, list of (scenario dict, seed))"""
    syn = importlib.import_module("necsim-rust_b200.synthetic")
    if name == "c4":
        return ("256 x SpatiallyImplicit sweep: J=floor(10^U(3,6)) deme 1, meta 1e7 deme 1, "
                "migration U(0.01,0.2), speciation 10^U(-6,-3), seeds 0..255", syn.config4())
    if name == "c4-small":
        # every 16th simulation of the sweep: the profiling-sized case
        return ("16 of the 256 SpatiallyImplicit sweep simulations (every 16th)",
                syn.config4()[::16])
    if name == "c5":
        d, s = syn.config5()
        return ("SpatiallyExplicit 128x128 habitat (0 w.p. 0.2 else U{1..500}), dense "
                "16384^2 Gaussian sigma=4 dispersal, speciation 1e-6, seed %d" % s, [(d, s)])
    if name == "c3":
        d, s = syn.config3()
        return ("SpatiallyExplicit 64x64 habitat, dense 4096^2 dispersal, speciation 1e-4, seed 1",
                [(d, s)])
    if name == "c2":
        d, s = syn.config2()
        return ("AlmostInfinite circle r=100, Normal sigma=10, speciation 1e-5, seed 7", [(d, s)])
    d, s = syn.config1()
    return ("NonSpatial 100x100 deme 10, speciation 1e-3, seed 42", [(d, s)])


# ---------------------------------------------------------------------------
# distributed plumbing (replicas only)
# ---------------------------------------------------------------------------
class Dist:
    """One process per GPU (torchrun env); replicas only: the process group
    carries the max-over-ranks time and the sum of events, never lineages.
    `backend="gloo"` runs the same plumbing on CPU tensors (tests)."""

    def __init__(self, backend="nccl", timeout_s=600):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.torch = None
        self.device = "cpu"
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as td
            self.torch = torch
            self.td = td
            if backend == "nccl":
                torch.cuda.set_device(self.local_rank)
                self.device = "cuda"
                td.init_process_group("nccl", timeout=datetime.timedelta(seconds=timeout_s),
                                      device_id=torch.device("cuda", self.local_rank))
            else:
                td.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))

    def barrier(self):
        if self.torch is not None:
            self.td.barrier()

    def max(self, v):
        if self.torch is None:
            return v
        t = self.torch.tensor([float(v)], dtype=self.torch.float64, device=self.device)
        self.td.all_reduce(t, op=self.td.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v):
        if self.torch is None:
            return v
        t = self.torch.tensor([float(v)], dtype=self.torch.float64, device=self.device)
        self.td.all_reduce(t, op=self.td.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.torch is not None:
            self.td.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            import tempfile
            fd, self.path = tempfile.mkstemp(prefix="necsim_clocks_%d_" % self.gpu, suffix=".csv")
            self.f = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        with open(self.path) as f:
            lines = f.readlines()
        try:
            os.unlink(self.path)
        except OSError:
            pass
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU restatement of the reference (bounded sample)
# ---------------------------------------------------------------------------
def cpu_partitions(n_sims, threads):
    """IsolatedIndividuals partitions per simulation: one when the workload
    has a simulation per thread, else enough to occupy every thread, as the
    reference spreads one simulation over cores (pre_sampler.rs:103-112)."""
    return max(1, threads // max(n_sims, 1))


def cpu_sample(sims, pause, threads, sampler="poisson", counts=None):
    """Runs the reference-faithful CPU restatement on every simulation of the
    workload up to time `pause` (a bounded sample), `threads` at a time, each
    simulation split into cpu_partitions() IsolatedIndividuals partitions.
    Returns (events, seconds); `counts`, when given, receives the sample's
    WyHash primes and draws (the reference's hash work for those events)."""
    import oracle
    code = oracle.SAMPLER_EXP if sampler == "exp" else oracle.SAMPLER_POISSON
    parts = cpu_partitions(len(sims), threads)
    tasks = [(d, seed, r) for d, seed in sims for r in range(parts)]

    def one(item):
        d, seed, rank = item
        o = oracle.simulate(d, seed, mode=oracle.MODE_REFERENCE, pause_before=pause, event_time_sampler=code,
                            partition=(rank, parts))
        return o.steps, o.n_primes, o.n_draws

    oracle.lib()
    t0 = time.perf_counter()
    with concurrent.futures.ThreadPoolExecutor(max_workers=threads) as ex:
        res = list(ex.map(one, tasks))
    if counts is not None:
        counts["steps"] = sum(r[0] for r in res)
        counts["primes"] = sum(r[1] for r in res)
        counts["draws"] = sum(r[2] for r in res)
    return sum(r[0] for r in res), time.perf_counter() - t0


def cpu_sample_desc(name, pause, n, threads=1):
    parts = cpu_partitions(n, threads)
    split = (", each in %d IsolatedIndividuals partitions" % parts) if parts > 1 else ""
    horizon = "to completion" if pause is None else "advanced to t=%g (pause_before)" % pause
    return "%s: all %d simulation(s) %s with the reference schedule%s" % (name, n, horizon, split)


def reference_arm(args, dist):
    if dist.rank != 0:
        dist.close()
        return
    desc, sims = workload(args.workload)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_sample(sims, args.cpu_sample_pause, threads, args.event_time_sampler)
    ev, sec = 0, 0.0
    for _ in range(args.steps):
        e, s = cpu_sample(sims, args.cpu_sample_pause, threads, args.event_time_sampler)
        ev += e
        sec += s
    value = ev / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+u64",
        "data": "synthetic", "config": {"workload": desc, "schedule": "reference Monolithic",
                                        "event_time_sampler": args.event_time_sampler},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": cpu_sample_desc(args.workload, args.cpu_sample_pause,
                                                   len(sims), threads)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    dist.close()


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def train_lifetime_model(nb, syn, device, pause):
    """The learned scheduler's model, trained before anything is timed on
    traces the backend generates from the AlmostInfinite circle (r = 100,
    sigma = 10) and the SpatiallyExplicit 64x64 landscape, each over a
    sweep of speciation probabilities, and a SpatiallyImplicit sweep, every
    run paused at `pause` (None: to completion; a paused run labels only the
    lineages that end before the pause, so long lives go unseen)."""
    ai, _ = syn.config2()
    se, _ = syn.config3()
    X, y = [], []
    t0 = time.perf_counter()
    for desc in (ai, se):
        nus = [1e-2, 1e-3, 1e-4]
        xs, ys = nb.collect_traces([syn.to_scenario(desc)] * len(nus), nus, [11, 12, 13],
                                   nb.CUDA(device=device), pause_before=pause, snapshot_rounds=16,
                                   max_rows=1 << 17)
        X.append(xs)
        y.append(ys)
    # SpatiallyImplicit traces from two sweeps of the same family with other
    # parameters (sweep seeds 99 and 98, speciation raised 100- and 10-fold
    # so that the runs end quickly)
    for sweep_seed, factor in ((99, 100.0), (98, 10.0)):
        si = syn.config4(n_sims=64, sweep_seed=sweep_seed)
        xs, ys = nb.collect_traces([syn.to_scenario(d) for d, _ in si],
                                   [d["speciation_probability"] * factor for d, _ in si],
                                   [1000 + s for _, s in si], nb.CUDA(device=device), pause_before=pause,
                                   snapshot_rounds=4, max_rows=1 << 17)
        X.append(xs)
        y.append(ys)
    X = np.concatenate(X)
    y = np.concatenate(y)
    model = nb.LifetimeModel(seed=1, device=device)
    losses = model.train(X, y, epochs=8, batch=1024, lr=2e-3, seed=3)
    info = {"trace_rows": int(X.shape[0]), "epochs": 8, "final_loss": float(losses[-1]),
            "label_variance": float(np.var(y)), "seconds": time.perf_counter() - t0,
            "traces": "AlmostInfinite r=100 sigma=10 and SpatiallyExplicit 64x64, speciation "
                      "{1e-2,1e-3,1e-4}, and two SpatiallyImplicit sweeps of 64 simulations (seeds 99 and "
                      "98, speciation x100 and x10), " + ("to completion" if pause is None else
                                                         "paused at t=%g" % pause)}
    return model, info


def canonical_work(sims, algo, pause, threads, sampler):
    """WyHash primes and draws per event of the canonical schedule -- the one
    the kernels execute -- counted by the oracle on every k-th simulation of
    the workload (at most 32) up to time `pause`, with the run's step_slice."""
    import oracle
    code = oracle.SAMPLER_EXP if sampler == "exp" else oracle.SAMPLER_POISSON
    pick = sims[:: max(1, len(sims) // 32)]

    def one(item):
        d, seed = item
        o = oracle.simulate(d, seed, mode=oracle.MODE_CANONICAL, pause_before=pause, event_time_sampler=code,
                            step_slice=algo.step_slice, min_round_events=algo.min_round_events,
                            step_slice_max=algo.step_slice_max)
        return o.steps, o.n_primes, o.n_draws

    oracle.lib()
    with concurrent.futures.ThreadPoolExecutor(max_workers=threads) as ex:
        res = list(ex.map(one, pick))
    return {"steps": sum(r[0] for r in res), "primes": sum(r[1] for r in res), "draws": sum(r[2] for r in res),
            "sample": "%d of %d simulation(s) to t=%g" % (len(pick), len(sims), pause)}


# DRAM bytes (read + write) per executed event of the round kernels (the
# cooperative kernel and the step kernel), from ncu captures of every launch
# of `bench.py --workload <w> --once` (dram__bytes_read.sum +
# dram__bytes_write.sum of those kernels / the run's events): the sweep's
# figure is the 16-simulation sweep's to t = 3000, scaled by events
DRAM_BYTES_PER_EVENT = {"c4": 1.95, "c4-small": 1.95, "c3": 36.5}


def issue_roofline(nb, device, work, events, kernel_ms, launches, workload_name):
    """The round kernels (the cooperative kernel and the step kernel, timed
    together by CUDA events around each round's launches) against their
    integer-issue bound: algorithmic WyHash mixing work per event -- wymum,
    the 64x64 -> 128-bit multiply-fold; a prime costs 2, a draw 1 -- on the
    canonical schedule, times the events, over the kernels' time, against
    the measured rate of independent wymum chains on this GPU."""
    per_event = (2.0 * work["primes"] + work["draws"]) / max(work["steps"], 1)
    achieved = per_event * events / (kernel_ms / 1e3) if kernel_ms > 0 else 0.0
    peak = nb.hash_peak(device)
    bpe = DRAM_BYTES_PER_EVENT.get(workload_name)
    return {"bound": "integer-issue", "achieved": achieved, "peak": peak, "unit": "wymum/s",
            "frac": achieved / peak,
            "traffic": (bpe * events / max(launches, 1)) if bpe else None,
            "traffic_unit": "DRAM bytes per launch (ncu per-event figure x events per launch)",
            "kernel": "coop_kernel + step_kernel", "avg_launch_ms": kernel_ms / max(launches, 1),
            "launches": launches, "wymum_per_event": per_event,
            "primes_per_event": work["primes"] / max(work["steps"], 1),
            "draws_per_event": work["draws"] / max(work["steps"], 1),
            "peak_source": "measured: 8 independent wymum chains per thread on every SM "
                           "(necsim_gpu_hash_peak)",
            "work_source": "canonical-schedule oracle, " + work["sample"]}


def roofline_entry(nb, device, sims, algo, pause, threads, sampler, events, kernel_ms, launches, name):
    """The `roofline` key: the canonical-schedule work count and the
    integer-issue roofline, or the error that prevented them (never fatal to
    the benchmark line)."""
    try:
        work = canonical_work(sims, algo, pause, threads, sampler)
        return issue_roofline(nb, device, work, events, kernel_ms, launches, name)
    except Exception as e:
        return {"error": "%s: %s" % (type(e).__name__, e)}


def host_cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def secondary(nb, name, pause, device, threads, sampler, note):
    """One secondary workload: the plain kernel's device time on the GPU
    (one warm-up run, one timed) beside the CPU restatement of the reference
    on the same horizon, `threads` at a time."""
    desc, sims = workload(name)
    syn = importlib.import_module("necsim-rust_b200.synthetic")
    scen = [syn.to_scenario(d) for d, _ in sims]
    algo = nb.CUDA(device=device, event_time_sampler=sampler)
    with nb.Batch(scen, [d["speciation_probability"] for d, _ in sims], [s for _, s in sims], algo,
                  pause_before=pause) as batch:
        batch.run()
        outs = batch.run()
    ev = sum(o.steps for o in outs)
    ms = outs[0].total_ms
    cev, csec = cpu_sample(sims, pause, threads, sampler)
    # the oracle builds its alias tables inside every run (the GPU time above
    # excludes the library's build): time one build alone and take it out
    import oracle
    t0 = time.perf_counter()
    oracle.build_alias(sims[0][0])
    build = time.perf_counter() - t0
    csec = max(csec - build, 1e-9)
    return {"workload": desc, "pause_before": pause, "value": ev / (ms / 1e3), "unit": UNIT,
            "ms": ms, "events": ev, "species": int(sum(o.biodiversity for o in outs)),
            "cpu_baseline": {"value": cev / csec, "unit": UNIT, "cores": threads, "kind": "port",
                             "seconds": csec, "table_build_seconds_excluded": build, "events": cev,
                             "cpu_model": host_cpu_model(),
                             "sample": cpu_sample_desc(name, pause, len(sims), threads) + note}}


def time_arm(nb, scen, nus, seeds, algo, args, dist):
    """Device-timed runs of a resident batch: warm-up, then `steps` runs."""
    batch = nb.Batch(scen, nus, seeds, algo, pause_before=args.pause)
    for _ in range(args.warmup):
        batch.run()
    dist.barrier()
    r = {"steps": 0, "dev_ms": 0.0, "kernel_ms": 0.0, "resident_ms": 0.0, "step_launches": 0, "visits": 0,
         "launches": 0, "n_spec": 0, "outs": None, "priority": batch.priority}
    for _ in range(args.steps):
        outs = batch.run()
        o0 = outs[0]
        r["steps"] += sum(o.steps for o in outs)
        r["n_spec"] += sum(o.n_speciation for o in outs)
        r["dev_ms"] += o0.total_ms          # device time of the whole batch (CUDA events)
        r["kernel_ms"] += o0.kernel_ms      # step-kernel time (CUDA events around each launch)
        r["resident_ms"] += o0.resident_ms  # resident-kernel time (its own stream, overlaps)
        r["step_launches"] += o0.n_step_launches
        r["visits"] += o0.lineage_visits
        r["launches"] += o0.n_launches
        r["outs"] = outs
    dist.barrier()
    batch.close()
    return r


def main():
    args = parse()
    dist = Dist()
    if args.impl == "reference":
        return reference_arm(args, dist)

    nb = importlib.import_module("necsim-rust_b200")
    syn = importlib.import_module("necsim-rust_b200.synthetic")
    desc, sims = workload(args.workload)
    scen = [syn.to_scenario(d) for d, _ in sims]
    nus = [d["speciation_probability"] for d, _ in sims]
    seeds = [s for _, s in sims]
    device = dist.local_rank if dist.world > 1 else 0
    # batches: simulations down to 8 lineages (one per warp of a resident
    # block) continue in the resident kernel on a stream of their own,
    # decoupled from the global rounds
    resident = True if len(sims) > 1 else False
    if args.once:
        with nb.Batch(scen, nus, seeds, nb.CUDA(device=device, event_time_sampler=args.event_time_sampler,
                                                resident=resident), pause_before=args.pause) as b:
            outs = b.run()
        print(json.dumps({"workload": args.workload, "pause_before": args.pause, "resident": resident,
                          "events": sum(o.steps for o in outs), "ms": outs[0].total_ms,
                          "rounds": outs[0].n_step_launches}), flush=True)
        dist.close()
        return
    se = sims[0][0]["kind"] == 3
    kind = sims[0][0]["kind"]

    model, model_info = None, None
    if args.schedule in ("learned", "both"):
        model, model_info = train_lifetime_model(nb, syn, device, args.train_pause)
    plain_algo = nb.CUDA(device=device, event_time_sampler=args.event_time_sampler, resident=resident)
    tune_info = None
    if args.autotune == "on" or (args.autotune == "auto" and args.workload.startswith("c4")):
        t0 = time.perf_counter()
        plain_algo, res = nb.autotune(scen, nus, seeds, plain_algo, sample_pause=400.0)
        tune_info = {"block_size": plain_algo.block_size, "step_slice": plain_algo.step_slice,
                     "dedup_factor_pct": plain_algo.dedup_factor_pct, "candidates": int(len(res)),
                     "sample": "every k-th simulation up to 4M origins, paused at t=400",
                     "seconds": time.perf_counter() - t0}
    head_algo = nb.CUDA(**{**plain_algo.__dict__, "schedule": "learned", "model": model}) if model else plain_algo

    plain = time_arm(nb, scen, nus, seeds, plain_algo, args, dist) if args.schedule == "both" else None
    clocks = Clocks(dist.local_rank)
    clocks.start()
    head = time_arm(nb, scen, nus, seeds, head_algo, args, dist)
    clk = clocks.stop()

    # end to end through the public C ABI with host buffers
    e2e_steps, e2e_sec, h2d, d2h = 0, 0.0, 0, 0
    for _ in range(args.steps):
        dist.barrier()
        t0 = time.perf_counter()
        outs = nb.simulate_batch(scen, nus, seeds, head_algo, pause_before=args.pause)
        dt = time.perf_counter() - t0
        e2e_sec += dist.max(dt)
        e2e_steps += sum(o.steps for o in outs)
        h2d += outs[0].h2d_bytes
        d2h += outs[0].d2h_bytes

    # where the end-to-end call's host time goes: the same batch set up
    # (engines, buffers, origins, CUDA graphs, model scores), run (device time
    # inside) and released, each timed on the host once
    t0 = time.perf_counter()
    bb = nb.Batch(scen, nus, seeds, head_algo, pause_before=args.pause)
    t1 = time.perf_counter()
    bo = bb.run()
    t2 = time.perf_counter()
    bb.close()
    t3 = time.perf_counter()
    e2e_parts = {"prepare_s": t1 - t0, "run_s": t2 - t1, "device_ms": bo[0].total_ms, "release_s": t3 - t2}

    max_ms = dist.max(head["dev_ms"])
    total_steps = dist.sum(head["steps"])
    value = total_steps / (max_ms / 1e3)
    e2e_value = dist.sum(e2e_steps) / e2e_sec
    steps, visits, n_spec = head["steps"], head["visits"], head["n_spec"]
    outs = head["outs"]

    # the round kernels against HBM (a secondary view: they are issue- and
    # latency-bound): algorithmic bytes = lineage state read and written per
    # visit (4 u32 + 5 u64/f64 + 1 flag, 57 B each way), speciation events
    # written (40 B) and, for SpatiallyExplicit, one 32-B cell record and one
    # 32-B atom sector per event
    # The round kernels' rooflines need every event to run in them: with the
    # resident kernel on they come from one more run with it off.
    r_steps, r_visits, r_spec = steps, visits, n_spec
    r_kernel_ms, r_launches = head["kernel_ms"], head["step_launches"]
    roof_note = "the timed runs"
    if resident:
        with nb.Batch(scen, nus, seeds, nb.CUDA(**{**plain_algo.__dict__, "resident": False}),
                      pause_before=args.pause) as b:
            b.run()
            ro = b.run()
        r_steps, r_spec = sum(o.steps for o in ro), sum(o.n_speciation for o in ro)
        r_visits, r_kernel_ms, r_launches = ro[0].lineage_visits, ro[0].kernel_ms, ro[0].n_step_launches
        roof_note = "one run with the resident kernel off (every event in the round kernels)"
    state_bytes = 2 * 57
    alg_bytes = r_visits * state_bytes + r_spec * 40 + (r_steps * 64 if se else 0)
    avg_launch_ms = r_kernel_ms / max(r_launches, 1)
    per_launch_bytes = alg_bytes / max(r_launches, 1)
    achieved = per_launch_bytes / (avg_launch_ms / 1e3) / 1e9 if avg_launch_ms > 0 else 0.0
    peak, peak_kind = load_peaks()

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+u64",
        "data": "synthetic",
        "config": {"workload": desc, "schedule": "learned" if model else "plain",
                   "resident": resident, "kind": kind,
                   "pause_before": args.pause, "event_time_sampler": args.event_time_sampler,
                   "simulations": len(sims), "lineages": int(sum(o.n_initial for o in outs)),
                   "l2": "inputs larger than L2 (lineage state %.2f GB)" % (
                       sum(o.n_initial for o in outs) * 57 * 2 / 1e9),
                   "parallelism": "replicas" if dist.world > 1 else "single"},
        "events_per_step": steps / args.steps,
        "clocks": clk,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d / args.steps,
                "d2h_bytes_per_step": d2h / args.steps, "parts": e2e_parts},
        "gpu_launches": head["launches"],
        "hbm_roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
                         "kernel": "coop_kernel + step_kernel", "avg_launch_ms": avg_launch_ms,
                         "launches": r_launches, "round_kernels_ms": r_kernel_ms, "timed": roof_note},
        # the per-simulation resident kernel runs the small simulations' rounds
        # on a second stream: a latency-bound chain of dependent 64-bit hash
        # multiplies per lineage, not a bandwidth roofline
        "resident": {"kernel": "resident_kernel", "ms_per_step": head["resident_ms"] / args.steps,
                     "share_of_step": head["resident_ms"] / max(head["dev_ms"], 1e-9)},
    }
    if plain is not None:
        p_ms = dist.max(plain["dev_ms"])
        p_value = dist.sum(plain["steps"]) / (p_ms / 1e3)
        same = all((a.steps, a.biodiversity, a.n_speciation, a.n_dedup, a.time) ==
                   (b.steps, b.biodiversity, b.n_speciation, b.n_dedup, b.time)
                   for a, b in zip(plain["outs"], head["outs"]))
        line["plain"] = {"value": p_value, "unit": UNIT, "ms_per_step": p_ms / args.steps,
                         "gpu_launches": plain["launches"]}
        line["learned_over_plain"] = value / p_value
        line["priority_sims"] = head["priority"]
        line["outcomes_identical"] = bool(same)
    # when each simulation ended on the device clock (from the batch's first
    # round): the priority engine's simulations against the others'
    prio = set(head["priority"])
    ends = [(o.end_ms, j) for j, o in enumerate(outs)]
    longest = max(ends)[1]
    line["timeline"] = {
        "batch_ms": outs[0].total_ms,
        "priority_last_end_ms": max((e for e, j in ends if j in prio), default=None),
        "others_last_end_ms": max((e for e, j in ends if j not in prio), default=None),
        "last_simulation": {"sim": longest, "end_ms": outs[longest].end_ms,
                            "routed_ms": outs[longest].routed_ms, "in_priority_engine": longest in prio},
        "priority_simulations": [{"sim": j, "routed_ms": outs[j].routed_ms, "end_ms": outs[j].end_ms}
                                 for j in head["priority"]],
    }
    if model_info is not None:
        line["model"] = model_info
    if tune_info is not None:
        line["autotune"] = tune_info
    threads = os.cpu_count() or 1
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        ev, sec = cpu_sample(sims, args.cpu_sample_pause, threads, args.event_time_sampler)
        line["cpu_baseline"] = {"value": ev / sec, "unit": UNIT, "cores": threads, "kind": "port",
                                "cpu_model": host_cpu_model(),
                                "sample": cpu_sample_desc(args.workload, args.cpu_sample_pause,
                                                          len(sims), threads)}
    # the same slice the CPU baseline and the reference arm time: every
    # simulation advanced to t = cpu_sample_pause, on the GPU (device time)
    if dist.world == 1 and args.pause is None:
        with nb.Batch(scen, nus, seeds, plain_algo, pause_before=args.cpu_sample_pause) as b:
            b.run()
            so = b.run()
        line["same_slice"] = {"value": sum(o.steps for o in so) / (so[0].total_ms / 1e3), "unit": UNIT,
                              "pause_before": args.cpu_sample_pause, "events": sum(o.steps for o in so),
                              "ms": so[0].total_ms, "schedule": "plain"}
    line["roofline"] = roofline_entry(nb, device, sims, plain_algo, args.cpu_sample_pause, threads,
                                      args.event_time_sampler, r_steps, r_kernel_ms, r_launches,
                                      args.workload)
    line["roofline"]["timed"] = roof_note
    if dist.rank == 0 and dist.world == 1 and args.workload == "c4" and not args.no_secondary:
        def guarded(*a):
            try:
                return secondary(*a)
            except Exception as e:  # a secondary never costs the headline line
                return {"error": "%s: %s" % (type(e).__name__, e)}
        line["secondary"] = {
            "c3": guarded(nb, "c3", None, device, threads, args.event_time_sampler, ""),
            # one thread: every oracle partition would build its own 5 GB alias table
            "c5_t400": guarded(nb, "c5", 400.0, device, 1, args.event_time_sampler, ""),
        }
    if model is not None:
        model.close()
    if dist.rank == 0:
        print(json.dumps(line), flush=True)
    dist.close()


if __name__ == "__main__":
    main()
