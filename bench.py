"""Benchmark: ns/day of the B200 step engine on the headline workload.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--config NAME] [--impl mdb|reference]

One "step" is one MD step (forces + LFMiddle + constraints) of the whole
workload.  With N > 1 (torchrun, one process per GPU) every rank advances its
own independent replica -- the step loop does not shard (replicas only) -- and
`value` is the sum over ranks, timed as the max over ranks.

Timing: W untimed warm-up steps, then exactly K steps replayed as CUDA-graph
strides of `--stride` steps, each stride timed with CUDA events recorded on the
engine's own stream; L2 (126 MB) is flushed between strides by writing a
256 MB buffer, outside the timed intervals.  `e2e` is the same metric through
the public Python API with host buffers: the state is uploaded from host memory
and positions are read back after every stride, wall-clock timed.

`--impl reference` times the reference's own CPU path on the host cores.  The
reference's CPU path is TypeScript, which cannot run here (no Node), so the
f64 C++ restatement of it (oracle/) stands in, with every host thread.
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "making-it-rain-webgpu_b200"))
sys.path.insert(0, str(ROOT))

TIME_STEP_PS = 0.002
NS_PER_DAY_PER_STEP_PER_S = TIME_STEP_PS * 86400 / 1000.0
# Algorithmic FP32 work per unique in-cutoff pair: 74 flop (FMA = 2, special
# functions = 1), the tally written down with the roofline in DESIGN.md.
FLOP_PER_PAIR = 74.0
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # nominal FP32 FMA issue rate at max SM clock


def workload(name: str, seed: int):
    from mdb200 import synth

    if name == "water-2652":
        s, st = synth.config_water_2652(seed=seed)
        return s, st, {"workload": "TIP3P water box, 2,652 atoms, 3.0 nm cube, PME 1.0 nm, mesh 30^3",
                       "atoms": s.particle_count}
    if name == "peptide-12k":
        s, st = synth.config_peptide_12k(seed=seed)
        return s, st, {"workload": "Ala20 helix ff14SB + caps, 5.0 nm TIP3P cube, 0.15 M NaCl, HBond SHAKE, "
                                   "PME 1.0 nm, mesh 50^3", "atoms": s.particle_count}
    if name == "octa-27k":
        s, st = synth.config_octahedron_27k(seed=seed)
        return s, st, {"workload": "60-residue (AGKE)15 chain ff14SB, TIP3P truncated octahedron, 0.15 M NaCl",
                       "atoms": s.particle_count}
    raise SystemExit(f"unknown --config {name}")


def default_config() -> str:
    from mdb200 import synth

    return "peptide-12k" if hasattr(synth, "config_peptide_12k") else "water-2652"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, start: float, end: float) -> dict:
        """Samples taken between `start` and `end` (perf_counter seconds)."""
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for stamp, line in self.lines:
            if not start <= stamp <= end:
                continue
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[3:7]):
                if flag.lower() in ("active", "1"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        loaded = [v for v in sm if v > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def flush_l2(buffer) -> None:
    buffer.zero_()


def cpu_time_oracle(system, state, steps_hint: int, budget_s: float, threads: int):
    """Steps/s of the f64 CPU restatement (oracle/), a bounded sample."""
    from oracle import oracle as orc

    t = time.perf_counter()
    p, v, step = orc.run(system, state, 1, seed=1, threads=threads)
    one = time.perf_counter() - t
    n = max(1, min(steps_hint, int(budget_s / max(one, 1e-6))))
    from mdb200.system import State

    st = State(positions=p, box=state.box, velocities=v, step=step)
    t = time.perf_counter()
    orc.run(system, st, n, seed=1, threads=threads)
    elapsed = time.perf_counter() - t
    return n / elapsed, n, elapsed


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=12000)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--stride", type=int, default=100)
    ap.add_argument("--config", default=None)
    ap.add_argument("--impl", default="mdb", choices=("mdb", "reference"))
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    config = args.config or default_config()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        system, state, cfg = workload(config, seed=1)
        threads = os.cpu_count() or 1
        sps, n, elapsed = cpu_time_oracle(system, state, args.steps, min(args.cpu_budget * 6, 240.0), threads)
        value = sps * NS_PER_DAY_PER_STEP_PER_S
        print(json.dumps({
            "impl": "reference", "metric": "ns/day", "value": value, "unit": "ns/day", "n_gpus": args.gpus,
            "steps": n, "warmup": 1, "ms_per_step": 1000.0 / sps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {**cfg, "parallelism": "host threads", "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": value, "unit": "ns/day", "cores": threads, "kind": "port",
                             "sample": f"{n} full MD steps of the same workload (f64 C++ restatement of "
                                       f"src/reference; the TypeScript original needs Node, absent here)"},
            "e2e": {"value": value, "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return

    import torch

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from mdb200 import steploop

    system, state, cfg = workload(config, seed=1 + rank)
    opts = steploop.RunOptions(seed=7 + rank, device=local, max_batch=args.stride)
    loop = steploop.StepLoop.from_parsed(system, state, opts)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    # clocks are sampled from before the warm-up, so nvidia-smi is running when
    # the timed region starts; only samples inside that region are reported
    clocks = ClockSampler(local).__enter__()
    # warm-up: graphs for the stride and the remainder, lists, clocks
    loop.run(args.warmup)
    stride = min(args.stride, args.steps)
    strides = [stride] * (args.steps // stride) + ([args.steps % stride] if args.steps % stride else [])
    for s in set(strides):
        loop.run(s)

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize()

    barrier()
    device_ms = 0.0
    timed_start = time.perf_counter()
    for s in strides:
        flush_l2(flush)
        torch.cuda.synchronize()
        device_ms += loop.run_timed(s)
    barrier()
    timed_end = time.perf_counter()
    time.sleep(0.3)  # let the sampler flush the last line of the region
    clocks.__exit__(None, None, None)
    total_s = device_ms / 1000.0
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([total_s], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_s = float(t.item())
    steps_per_s = args.steps / total_s
    value = steps_per_s * NS_PER_DAY_PER_STEP_PER_S * world

    # end to end through the public API, host buffers in and out
    n = system.particle_count
    host_pos = np.ascontiguousarray(state.positions, dtype=np.float64)
    host_vel = np.ascontiguousarray(state.velocities, dtype=np.float64)
    barrier()
    t0 = time.perf_counter()
    loop.set_positions(host_pos)
    loop.set_velocities(host_vel)
    readbacks = 0
    for s in strides:
        loop.run(s)
        out = loop.positions()
        readbacks += 1
    e2e_s = time.perf_counter() - t0
    barrier()
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([e2e_s], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = args.steps / e2e_s * NS_PER_DAY_PER_STEP_PER_S * world
    assert np.isfinite(out).all()

    # stage profile for the roofline (advances the replica; done after timing)
    prof = loop.profile_step(repeats=20)
    pairs = prof["pairs_within_cutoff"]
    nb_s = prof["ms_nonbonded"] / 1000.0
    achieved = FLOP_PER_PAIR * pairs / nb_s / 1e12
    peaks = {}
    peaks_path = ROOT / "MEASURED_PEAKS.json"
    if peaks_path.exists():
        peaks = json.loads(peaks_path.read_text())
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    mesh = prof["mesh_points"]
    atoms = prof["atoms"]
    spread_bytes = 28 * atoms + 8 * mesh
    gather_bytes = 4 * mesh + 52 * atoms
    integ_bytes = 124 * atoms
    stages = {
        "nonbonded_ms": prof["ms_nonbonded"], "listed_ms": prof["ms_listed"], "pme_ms": prof["ms_pme"],
        "pme_spread_ms": prof["ms_pme_spread"], "pme_fft_ms": prof["ms_pme_fft"],
        "pme_gather_ms": prof["ms_pme_gather"], "integrate_ms": prof["ms_integrate"],
        "list_check_ms": prof["ms_list_check"], "list_rebuild_ms": prof["ms_list_rebuild"],
        "step_ms": prof["ms_step"], "pairs_within_cutoff": pairs, "tiles": prof["tiles"],
        "pair_fraction_in_tiles": pairs / max(1, prof["tiles"] * 1024),
        "spread_GBs": spread_bytes / (prof["ms_pme_spread"] / 1000) / 1e9,
        "gather_GBs": gather_bytes / (prof["ms_pme_gather"] / 1000) / 1e9,
        "integrate_GBs": integ_bytes / (prof["ms_integrate"] / 1000) / 1e9,
    }

    result = {
        "metric": "ns/day", "value": value, "unit": "ns/day", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_s * 1000.0 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 pair math, int64 fixed-point accumulation",
        "data": "synthetic",
        "config": {**cfg, "time_step_ps": TIME_STEP_PS, "steps_per_s": steps_per_s * world,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": f"flushed (256 MB write) between timed strides of {stride} steps"},
        "e2e": {"value": e2e_value, "unit": "ns/day", "h2d_bytes_per_step": 48 * n / args.steps,
                "d2h_bytes_per_step": 24 * n * readbacks / args.steps},
        "gpu_launches": int(prof["launches_per_step"]) * args.steps,
        "roofline": {"bound": "fp32", "kernel": "k_nonbonded", "achieved": achieved, "peak": FP32_PEAK_TFLOPS,
                     "unit": "TFLOP/s", "frac": achieved / FP32_PEAK_TFLOPS, "traffic": None,
                     "peak_source": "nominal FP32 issue rate, 148 SM x 128 lanes x 2 flop x 1.965 GHz",
                     "algorithmic": f"{FLOP_PER_PAIR:.0f} flop x {pairs} in-cutoff pairs per launch",
                     "hbm_peak_gbs": hbm_peak, "stages": stages},
        "clocks": clocks.summary(timed_start, timed_end),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sps, nsteps, elapsed = cpu_time_oracle(system, state, 1000, args.cpu_budget, threads)
        result["cpu_baseline"] = {
            "value": sps * NS_PER_DAY_PER_STEP_PER_S, "unit": "ns/day", "cores": threads, "kind": "port",
            "sample": f"{nsteps} MD steps of the same workload in {elapsed:.1f} s (f64 C++ restatement of "
                      "src/reference, OpenMP over all host threads)"}
    loop.destroy()
    if rank == 0:
        print(json.dumps(result))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
