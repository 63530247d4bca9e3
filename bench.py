"""Benchmark of the B200 vertical advance (column-steps/s).

Workload (N=1): a whole 1 deg x 1 deg globe, 180 x 360 = 64,800 columns,
nAlts = 50, 6 neutral species, FP64, dt = 2 s: the batched, graph-captured
forward of the 1-degree configuration.  A "step" is one RK4 vertical step
(producers, gather, 4 stages, 5 boundary passes, scatter) of every column.
Inputs are seeded synthetic columns (gitm_b200/synthetic.py); the state
(about 0.9 GB) is larger than L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--solver rusanov|ausm]

The default solver is Rusanov (GITM's default, UseAUSMSolver = F); `--solver
ausm` measures the AUSM solver on the same workload.

Under torchrun (N > 1) every rank advances its own globe (an ensemble member
seeded by rank): weak scaling, no data exchange in the timed loop.
`--impl reference` times the CPU restatement of the reference (the oracle)
on the host cores on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import shutil
import subprocess
import tempfile
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "column-steps/s, 1 deg grid (64,800 columns x 50 alts, FP64 RK4 vertical step)"
UNIT = "column-steps/s"
DT = 2.0
CHUNK = 100  # steps per captured graph; the input state is restored between graphs


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--deg", type=float, default=1.0, help="grid spacing in degrees")
    ap.add_argument("--n-alts", type=int, default=50)
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--launch", default="", help="threads,steps_per_launch,ctas_per_sm (skips autotune)")
    ap.add_argument("--e2e-steps", type=int, default=4)
    ap.add_argument("--plain-steps", type=int, default=30)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--sustained", type=float, default=2.0,
                    help="seconds of device time of the sustained leg (0 = skip)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the AUSM, adjoint and ensemble legs of the default run")
    ap.add_argument("--extra-fd", type=int, default=4,
                    help="finite-difference directions of the adjoint leg of the default run")
    ap.add_argument("--solver", default="rusanov", choices=["rusanov", "ausm"])
    ap.add_argument("--adjoint", action="store_true",
                    help="measure the adjoint rollout (2.5 deg globe, 60 steps, checkpoint every 10)")
    ap.add_argument("--adj-steps", type=int, default=60)
    ap.add_argument("--adj-every", type=int, default=10)
    ap.add_argument("--adj-deg", type=float, default=2.5)
    ap.add_argument("--fd-directions", type=int, default=32)
    ap.add_argument("--ensemble", action="store_true",
                    help="measure the uneven ensemble: 48 members of mixed resolution and nAlts in one plan")
    ap.add_argument("--ens-members", type=int, default=48)
    ap.add_argument("--ens-steps", type=int, default=200)
    ap.add_argument("--ens-plain-steps", type=int, default=3)
    ap.add_argument("--horizontal", action="store_true",
                    help="measure the horizontal advance (advance_horizontal) on a globe of 9x9 blocks")
    ap.add_argument("--hz-deg", type=float, default=1.0)
    ap.add_argument("--hz-steps", type=int, default=50)
    return ap.parse_args()


SOLVER_NAMES = {"rusanov": "Rusanov RK4", "ausm": "AUSM RK4"}


def solver_params(name: str, **over):
    from gitm_b200 import abi
    return abi.default_params(solver=abi.SOLVER_AUSM if name == "ausm" else abi.SOLVER_RUSANOV, **over)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock, power and clock-event reasons sampled during a region.

    NVML (read-only queries) from a thread every 10 ms, so that even a short
    timed region has samples; nvidia-smi at 200 ms when NVML cannot be
    loaded.  The device is found by its PCI bus id, so the sample is of the
    GPU the process runs on whatever CUDA_VISIBLE_DEVICES says."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int, interval_s: float = 0.01):
        self.idx = device_index
        self.interval = interval_s
        self.samples = []
        self.thread = None
        self.proc = None
        self.nvml = None
        self.handle = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        self.nvml = pynvml
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.idx)
            bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.idx)

    def start(self):
        import threading
        try:
            self.handle = self._nvml_handle()
            self.smax = float(self.nvml.nvmlDeviceGetMaxClockInfo(self.handle, self.nvml.NVML_CLOCK_SM))
        except Exception:
            self.handle = None
        if self.handle is not None:
            self.stop_flag = threading.Event()

            def loop():
                n = self.nvml
                while not self.stop_flag.is_set():
                    try:
                        self.samples.append((float(n.nvmlDeviceGetClockInfo(self.handle, n.NVML_CLOCK_SM)),
                                             int(n.nvmlDeviceGetCurrentClocksEventReasons(self.handle)),
                                             n.nvmlDeviceGetPowerUsage(self.handle) / 1e3,
                                             n.nvmlDeviceGetTemperature(self.handle, n.NVML_TEMPERATURE_GPU)))
                    except Exception:
                        pass
                    self.stop_flag.wait(self.interval)
            self.thread = threading.Thread(target=loop, daemon=True)
            self.thread.start()
            return
        try:
            self.tmp = tempfile.mkdtemp(prefix="gitm_clocks_")
            self.path = os.path.join(self.tmp, "clocks.csv")
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}", "--format=csv,noheader",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            sm = [a for a, _, _, _ in self.samples]
            reasons = sorted({name for _, r, _, _ in self.samples for name, bit in self.REASONS if r & bit})
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax,
                    "sm_min_mhz": min(sm) if sm else None,
                    "reasons": reasons, "samples": len(sm),
                    "power_w_max": max((p for _, _, p, _ in self.samples), default=None),
                    "temp_c_max": max((t for _, _, _, t in self.samples), default=None),
                    "source": f"NVML every {1e3 * self.interval:g} ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no clock source"], "samples": 0}
        try:
            return self._read_smi()
        finally:
            shutil.rmtree(self.tmp, ignore_errors=True)

    def _read_smi(self) -> dict:
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1].split()[0]))
                smax.append(float(parts[2].split()[0]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi every 200 ms"}


# ---------------------------------------------------------------- helpers
def opcount(n_alts: int, solver: str = "rusanov") -> float:
    with open(os.path.join(ROOT, "tests", "golden", "opcount.json")) as f:
        d = json.load(f)
    return float(d[solver][str(n_alts)]["flop_eq_per_column_step"])


def profile_traffic():
    """DRAM bytes per column and launch of the step kernel (the state is read
    and written once per launch, whatever the steps per launch) from the
    committed ncu summary (profiles/vert_step_kernel_globe1deg.md), or None."""
    p = os.path.join(ROOT, "profiles", "vert_step_kernel_globe1deg.md")
    if not os.path.exists(p):
        return None
    m = re.search(r"dram_bytes_per_column_per_launch:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


def algorithmic_bytes_per_column_step(n_alts: int) -> float:
    """Compulsory HBM bytes of one launch per column (state read once, written
    once): reads NDensityS(6), IDensityS advected(2) + passive boundary cells,
    Rho, Temperature, Velocity(3), VerticalVelocity(6), IVelocity up, eddy;
    writes the same state, electrons, LogNS(6), NDensity."""
    G = n_alts + 4
    reads = (6 + 2 + 1 + 1 + 3 + 6 + 1 + 1) * G + 7 * G  # passive ions read for the e- sum
    writes = (6 + 2 + 1 + 1 + 1 + 3 + 6 + 6 + 1) * G + 7 * 11
    return 8.0 * (reads + writes)


def measure_fp64_peak(torch, device) -> float:
    """Dense FP64 GEMM throughput (cuBLAS DGEMM through torch), TFLOP/s."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(3):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def workload_name(deg: float, n_cols: int, n_alts: int, solver: str) -> str:
    """config.workload, the same string in both arms."""
    return f"globe {deg:g} deg, {n_cols} columns x {n_alts} alts, {SOLVER_NAMES[solver]}, dt 2 s"


def cpu_oracle_rates(m, seconds_per_call: float, n_calls: int, n_warm: int, solver: str = "rusanov",
                     threads: int | None = None):
    """The oracle (CPU restatement of the reference) on the host cores on a
    bounded sample of the workload: the first S columns, one RK4 step per
    call, S sized so that a call takes about seconds_per_call.  Every call
    advances a fresh copy made (and first touched) outside the timed region;
    n_warm untimed calls come first.  Returns the rates of the timed calls
    and a description of the sample.  The same procedure serves the
    cpu_baseline of our arm and the reference arm."""
    from gitm_b200.parallel import shard_member
    from oracle import oracle

    try:
        import torch
        torch.set_num_threads(1)  # torch's own CPU pool stays idle beside the oracle's threads
    except Exception:
        pass
    threads = threads or os.cpu_count() or 1
    p = solver_params(solver)
    probe = shard_member(m, 0, max(1, m.n_cols // (64 * threads)))
    work = probe.copy()
    t0 = time.perf_counter()
    oracle.advance(work, p, DT, 1, nthreads=threads)
    rate = probe.n_cols / max(time.perf_counter() - t0, 1e-6)
    n = int(min(m.n_cols, max(threads, rate * seconds_per_call)))
    sample = shard_member(m, 0, max(1, m.n_cols // n)) if n < m.n_cols else m
    rates, els = [], []
    for i in range(n_warm + n_calls):
        work = sample.copy()
        t0 = time.perf_counter()
        oracle.advance(work, p, DT, 1, nthreads=threads)
        el = time.perf_counter() - t0
        if i >= n_warm:
            rates.append(sample.n_cols / el)
            els.append(el)
    desc = (f"{sample.n_cols} of {m.n_cols} columns x 1 step (nAlts {m.n_alts}), C++ oracle -O3, "
            f"{threads} threads, median of {n_calls} calls of {statistics.median(els):.2f} s after "
            f"{n_warm} untimed")
    return rates, desc, threads


def cpu_baseline(m, seconds: float, solver: str = "rusanov") -> dict:
    """cpu_baseline of our arm: the oracle on the host cores, one untimed
    call and five timed ones of about seconds / 5 each, the median."""
    rates, desc, threads = cpu_oracle_rates(m, max(seconds / 5.0, 0.5), 5, 1, solver)
    return {"value": statistics.median(rates), "unit": UNIT, "cores": threads, "kind": "port", "sample": desc}


# ---------------------------------------------------------------- reference arm
def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from gitm_b200 import synthetic

    m = synthetic.globe_member(args.deg, args.deg, n_alts=args.n_alts, seed=0)
    per_call = min(max(args.cpu_seconds / max(1, args.steps + args.warmup), 0.5), 2.0)
    rates, desc, threads = cpu_oracle_rates(m, per_call, max(args.steps, 1), args.warmup, args.solver)
    v = statistics.median(rates)
    cb = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc}
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * m.n_cols / v,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded)",
           "config": {"workload": workload_name(args.deg, m.n_cols, args.n_alts, args.solver),
                      "parallelism": "host threads"},
           "cpu_baseline": cb,
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


# ---------------------------------------------------------------- our arm
STATE_NAMES = ("ndensity_s", "idensity_s", "rho", "temperature", "velocity", "vert_vel")


class GraphSteps:
    """Graph-captured steps of a plan: a graph of `chunk` steps (and one of
    the remainder, so that exactly `steps` steps are timed), replayed with the
    member's input state restored between replays outside the timed region
    (a vertical-only column has no damping and its waves grow without the
    rest of GITM, so long runs time the same physical regime)."""

    def __init__(self, torch, plan, members, dev, steps: int, chunk: int = CHUNK):
        self.torch, self.plan, self.dev = torch, plan, dev
        self.snap = [{k: d.tensors[k].clone() for k in STATE_NAMES} for d in members]
        self.members = members
        self.chunk = min(steps, chunk)
        self.n_full, rem = divmod(steps, self.chunk)
        self.cap = torch.cuda.Stream(dev)
        self.cap.wait_stream(torch.cuda.current_stream(dev))
        self.graphs = [(self._capture(self.chunk), self.chunk)] * self.n_full
        if rem:
            self.graphs.append((self._capture(rem), rem))
        torch.cuda.synchronize()

    def _capture(self, n):
        g = self.torch.cuda.CUDAGraph()
        with self.torch.cuda.stream(self.cap):
            with self.torch.cuda.graph(g, stream=self.cap):
                self.plan.advance(DT, n, stream=self.cap)
        return g

    def restore(self):
        for d, sn in zip(self.members, self.snap):
            for k in STATE_NAMES:
                d.tensors[k].copy_(sn[k])

    def launches(self) -> int:
        return sum(self.plan.launch_count(n) for _, n in self.graphs)

    def run(self, graphs=None):
        """Device seconds of the replays (CUDA events on the capture stream)."""
        torch = self.torch
        el = 0.0
        for g, _ in (graphs or self.graphs):
            self.restore()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(self.cap):
                e0.record(self.cap)
                g.replay()
                e1.record(self.cap)
            e1.synchronize()
            el += e0.elapsed_time(e1) / 1e3
        return el

    def sustained(self, seconds: float, clocks):
        """Replays of the chunk graph for at least `seconds` of device time:
        (steps, device seconds, clock record)."""
        clocks.start()
        el, steps = 0.0, 0
        while el < seconds:
            el += self.run(self.graphs[:1])
            steps += self.graphs[0][1]
        return steps, el, clocks.stop()


def run_ours(args):
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    if world > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    from gitm_b200 import synthetic
    from gitm_b200 import vertical as V

    m = synthetic.globe_member(args.deg, args.deg, n_alts=args.n_alts, seed=rank)
    n_cols = m.n_cols
    p = solver_params(args.solver)
    ctx = V.VerticalContext(p, device=local)
    dm = V.device_member(m, device=dev)
    plan = V.Plan(ctx, [dm])

    # -- plain per-step drop-in (default launch shape, one synchronous call per step)
    plain = None
    if args.plain_steps > 0:
        V.advance_vertical_all(ctx, [dm], DT, 1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.plain_steps):
            V.advance_vertical_all(ctx, [dm], DT, 1)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        plain = {"value": n_cols * args.plain_steps / el, "unit": UNIT,
                 "ms_per_step": 1e3 * el / args.plain_steps,
                 "how": "gitm_vert_advance_native per step (plan built each call, 256 threads, "
                        "1 step per launch, synchronous), wall clock"}
        # restore the input state for the batched run
        dm = V.device_member(m, device=dev)
        plan.close()
        plan = V.Plan(ctx, [dm])

    # -- batched: autotuned launch shape, graph-captured steps
    if args.launch:
        t, spl, cps = (int(x) for x in args.launch.split(","))
        plan.set_config(threads=t, steps_per_launch=spl, ctas_per_sm=cps)
    elif not args.no_autotune:
        # tuned on the timed step count itself when it is short (its steps
        # per launch then divide it: 1, K/2 or K), else on 16 steps
        plan.autotune(DT, args.steps if args.steps <= 32 else 16)
    cfg = plan.config
    gs = GraphSteps(torch, plan, [dm], dev, args.steps)
    for _ in range(max(args.warmup, 1)):  # W untimed warm-up replays of the timed graphs
        gs.run(gs.graphs[:1])
    torch.cuda.synchronize()
    plan.check()
    launches = gs.launches()

    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    el = gs.run()
    torch.cuda.synchronize()
    clk = clocks.stop()
    steps_done = sum(n for _, n in gs.graphs)
    if world > 1:
        t = torch.tensor([el], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        el = float(t.item())
        dist.barrier()
    st, nbad = plan.status(clear=True)
    total_cs = n_cols * steps_done * world
    value = total_cs / el

    # -- the same replays for at least args.sustained seconds (clocks sampled)
    sus = None
    if args.sustained > 0:
        s_steps, s_el, s_clk = gs.sustained(args.sustained, ClockSampler(local))
        sus = {"value": n_cols * s_steps / s_el, "unit": UNIT, "steps": s_steps, "device_seconds": s_el,
               "clocks": s_clk, "how": "the timed graph replayed for >= %g s of device time" % args.sustained}
        st2, nb2 = plan.status(clear=True)
        st, nbad = st | st2, max(nbad, nb2)
    gs.restore()
    del gs

    # -- end to end through the host-pointer C ABI (pinned host buffers)
    e2e = e2e_opt = None
    if args.e2e_steps > 0:
        e2e = e2e_leg(torch, V, ctx, m, args.e2e_steps, world, dev, optional_outputs=False)
        e2e_opt = e2e_leg(torch, V, ctx, m, args.e2e_steps, world, dev, optional_outputs=True)

    if rank == 0:
        flops_cs = opcount(args.n_alts, args.solver)
        n_launch = max(1, launches)
        t_launch = el / n_launch
        cs_launch = n_cols * steps_done / n_launch
        fp64_peak = measure_fp64_peak(torch, dev)
        hbm_peak = None
        try:
            hbm_peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
        except Exception:
            pass
        bytes_cs = algorithmic_bytes_per_column_step(args.n_alts) / max(1, cfg.steps_per_launch)
        achieved = flops_cs * cs_launch / t_launch / 1e12
        traffic = profile_traffic() if args.solver == "rusanov" else None
        roof = {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak,
                "traffic": None if traffic is None else traffic * n_cols,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of the "
                                  "2 deg globe (profiles/vert_step_kernel_globe1deg.md), per column and "
                                  "launch, times the columns of a launch",
                "kernel": "vert_step_kernel",
                "peak_source": "FP64 DGEMM (cuBLAS via torch.matmul 8192^3) measured in this run "
                               "(MEASURED_PEAKS.json has no FP64 figure)",
                "flops_per_column_step": flops_cs,
                "flop_convention": "add/mul/div/sqrt = 1, exp/log/pow = 20 (oracle count, dead code excluded)"}
        hbm = None
        if hbm_peak:
            ach = bytes_cs * n_cols * steps_done / el / 1e9
            hbm = {"bound": "hbm", "achieved": ach, "peak": hbm_peak, "unit": "GB/s",
                   "frac": ach / hbm_peak, "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"}
        cb = cpu_baseline(m, args.cpu_seconds, solver=args.solver) if args.cpu_seconds > 0 else None
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
               "steps": steps_done, "warmup": args.warmup,
               "ms_per_step": 1e3 * el / steps_done, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
               "config": {"workload": workload_name(args.deg, n_cols, args.n_alts, args.solver),
                          "columns_per_gpu": n_cols, "n_alts": args.n_alts,
                          "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                          "l2": "state larger than L2 (no flush needed)",
                          "launch": {"threads": cfg.threads, "cols_per_cta": cfg.cols_per_cta,
                                     "steps_per_launch": cfg.steps_per_launch,
                                     "ctas_per_sm": cfg.ctas_per_sm, "graph": True,
                                     "graph_steps": min(args.steps, CHUNK),
                                     "state_restored_every": min(args.steps, CHUNK)}},
               "clocks": clk, "gpu_launches": launches, "status": {"or": st, "bad_columns": nbad},
               "roofline": roof, "roofline_hbm": hbm, "cpu_baseline": cb, "e2e": e2e,
               "e2e_with_optional_outputs": e2e_opt, "plain": plain, "sustained": sus}
    plan.close()
    del dm
    torch.cuda.empty_cache()
    if rank == 0:
        if world == 1 and not args.no_extras:
            out["extras"] = run_extras(args, m)
        print(json.dumps(out))
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def e2e_leg(torch, V, ctx, m, n_steps: int, world: int, dev, optional_outputs: bool) -> dict:
    """The same metric end to end through the host-pointer C ABI
    (gitm_vert_advance_native_host) with pinned host arrays: every step copies
    in the arrays advance_vertical reads, steps and copies out the state it
    writes (and LogNS / NDensity with optional_outputs); wall clock."""
    import torch.distributed as dist
    pinned = m.copy()
    # Gamma, MeanMajorMass, TempUnit and cMax are the device's own producers
    # here (compute_coefficients = 1), not copied
    pinned.gamma = pinned.mean_major_mass = pinned.temp_unit = pinned.cmax = None
    if not optional_outputs:
        pinned.log_ns = pinned.ndensity = None
    for name, arr in list(pinned.arrays()):
        t = torch.from_numpy(arr).pin_memory()
        setattr(pinned, name, t.numpy())
    ins = ("ndensity_s", "idensity_s", "rho", "temperature", "velocity", "vert_vel", "ivel_up", "eddy",
           "cos_lat", "sza", "mlat")
    outs = STATE_NAMES + (("log_ns", "ndensity") if optional_outputs else ())
    h2d = sum(getattr(pinned, k).nbytes for k in ins)
    d2h = sum(getattr(pinned, k).nbytes for k in outs)
    V.advance_vertical_all_host(ctx, [pinned], DT, 1)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    calls = []
    for _ in range(n_steps):
        c0 = time.perf_counter()
        V.advance_vertical_all_host(ctx, [pinned], DT, 1)  # returns with the copies out done
        calls.append(time.perf_counter() - c0)
    torch.cuda.synchronize()
    ee = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([ee], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ee = float(t.item())
    return {"value": m.n_cols * n_steps * world / ee, "unit": UNIT,
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "call_ms": {"median": 1e3 * statistics.median(calls), "min": 1e3 * min(calls),
                        "max": 1e3 * max(calls)},
            "how": "gitm_vert_advance_native_host per step: the pinned host arrays advance_vertical "
                   "reads copied in, stepped, the state it writes copied out"
                   + (" with the optional LogNS and NDensity outputs" if optional_outputs else "")
                   + " (16 chunks, copies in / steps / copies out on three streams); wall clock"}


def ausm_report(args, m) -> dict:
    """The same globe and metric with the AUSM solver (UseAUSMSolver = T):
    autotuned launch shape, exactly args.steps graph-captured steps."""
    import torch

    from gitm_b200 import vertical as V
    dev = torch.device("cuda", torch.cuda.current_device())
    ctx = V.VerticalContext(solver_params("ausm"), device=dev.index)
    dm = V.device_member(m, device=dev)
    plan = V.Plan(ctx, [dm])
    plan.autotune(DT, min(args.steps, 8))
    cfg = plan.config
    gs = GraphSteps(torch, plan, [dm], dev, args.steps)
    gs.run(gs.graphs[:1])
    plan.check()
    clocks = ClockSampler(dev.index)
    clocks.start()
    el = gs.run()
    clk = clocks.stop()
    steps = sum(n for _, n in gs.graphs)
    launches = gs.launches()
    st, nbad = plan.status(clear=True)
    plan.close()
    ctx.close()
    flops = opcount(args.n_alts, "ausm")
    value = m.n_cols * steps / el
    return {"metric": "column-steps/s, AUSM solver", "value": value, "unit": UNIT, "steps": steps,
            "ms_per_step": 1e3 * el / steps,
            "config": {"workload": workload_name(args.deg, m.n_cols, args.n_alts, "ausm"),
                       "launch": {"threads": cfg.threads, "steps_per_launch": cfg.steps_per_launch,
                                  "ctas_per_sm": cfg.ctas_per_sm, "graph": True}},
            "roofline": {"bound": "fp64", "achieved": flops * value / 1e12, "unit": "TFLOP/s",
                         "flops_per_column_step": flops,
                         "how": "frac against the FP64 DGEMM peak of the main line"},
            "clocks": clk, "gpu_launches": launches, "status": {"or": st, "bad_columns": nbad}}


def run_extras(args, m) -> dict:
    """The rest of the reference's headline metric, measured in the default
    run: the AUSM solver on the same globe, the adjoint rollout (adjoint /
    forward cost, peak memory) and the uneven ensemble against the per-member
    plain loop.  Each is bounded to well under a minute of work."""
    out = {}
    for name, fn in (("ausm", lambda: ausm_report(args, m)),
                     ("adjoint", lambda: run_adjoint(args, fd_directions=args.extra_fd)),
                     ("ensemble", lambda: run_ensemble(args))):
        t0 = time.perf_counter()
        try:
            out[name] = fn()
        except Exception as exc:  # an extra that fails is reported, not fatal to the line
            out[name] = {"error": f"{type(exc).__name__}: {exc}"}
        if isinstance(out[name], dict):
            out[name]["wall_seconds"] = time.perf_counter() - t0
        __import__("torch").cuda.empty_cache()
    return out


# ---------------------------------------------------------------- adjoint
def run_adjoint(args, fd_directions: int | None = None):
    """Adjoint rollout: J = sum_c w_c log(n_O / n_N2) at 400 km after
    adj_steps steps of the adj_deg globe, w_c ~ U[0, 1]; gradients with
    respect to the initial state, the eddy coefficient and the per-column
    heating factor through gitm_b200.adjoint.rollout (checkpoints every
    adj_every steps).  Reports forward and backward device time, their ratio
    per step, the peak device memory and a finite-difference check.  Returns
    the report (rank 0) or None."""
    if fd_directions is None:
        fd_directions = args.fd_directions
    import torch

    from gitm_b200 import abi, synthetic
    from gitm_b200 import adjoint as AD
    from gitm_b200 import vertical as V

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    m = synthetic.globe_member(args.adj_deg, args.adj_deg, n_alts=args.n_alts, seed=rank, with_heating=True)
    n_cols = m.n_cols
    ctx = V.VerticalContext(abi.default_params(), device=local)
    run = AD.StepRunner(ctx, m, DT)
    base = run.state()
    eddy0 = run.tensors["eddy"].clone()
    hs0 = run.tensors["heating_scale"].clone()
    lvl = AD.level_of(m.altitude, 400e3)
    gen = torch.Generator(dev).manual_seed(11)
    w = torch.rand(n_cols, dtype=torch.float64, device=dev, generator=gen)
    names = ("ndensity_s", "temperature", "velocity", "vert_vel", "rho")

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def grads_once(n_steps, every=None):
        s0 = {k: v.clone().requires_grad_(True) for k, v in base.items()}
        ed = eddy0.clone().requires_grad_(True)
        hs = hs0.clone().requires_grad_(True)
        e0, e1, e2 = ev(), ev(), ev()
        e0.record()
        out = AD.rollout(run, s0, n_steps, args.adj_every if every is None else every, ed, hs)
        J = AD.o_n2_objective(out["ndensity_s"], w, lvl)
        e1.record()
        g = torch.autograd.grad(J, [s0[k] for k in names] + [ed, hs])
        e2.record()
        e2.synchronize()
        return g, e0.elapsed_time(e1) / 1e3, e1.elapsed_time(e2) / 1e3, float(J.detach())

    grads_once(args.adj_steps)  # warm-up at full length (plans, scratch, the saved-state buffers)
    clocks = ClockSampler(local)  # over every timed part of the leg
    clocks.start()
    # plain forward of the same rollout: one launch per step, no checkpoints
    torch.cuda.synchronize()
    f0, f1 = ev(), ev()
    f0.record()
    s = {k: v.clone() for k, v in base.items()}
    for _ in range(args.adj_steps):
        s = run.step(s, eddy0, hs0)
    f1.record()
    f1.synchronize()
    t_plain = f0.elapsed_time(f1) / 1e3
    free0 = torch.cuda.mem_get_info(dev)[0]
    torch.cuda.reset_peak_memory_stats(dev)
    # three timed rollouts, the median of each leg (the backward runs from
    # Python autograd, so host load on the machine shows in single runs)
    runs = [grads_once(args.adj_steps) for _ in range(3)]
    grads, _, _, Jv = runs[-1]
    t_fwd = statistics.median(r[1] for r in runs)
    t_bwd = statistics.median(r[2] for r in runs)
    peak_torch = torch.cuda.max_memory_allocated(dev)
    free1 = torch.cuda.mem_get_info(dev)[0]
    # the same rollout keeping every step's stage states from the forward
    # (every = 0: no recompute in the backward), where they fit
    kept = None
    if args.adj_steps * run.stage_bytes_per_step() < 0.8 * free1:
        grads_once(args.adj_steps, every=0)
        torch.cuda.reset_peak_memory_stats(dev)
        runs0 = [grads_once(args.adj_steps, every=0) for _ in range(3)]
        k_fwd = statistics.median(r[1] for r in runs0)
        k_bwd = statistics.median(r[2] for r in runs0)
        g0 = runs0[-1][0]
        agree = max(float((a - b).norm() / max(float(b.norm()), 1e-300)) for a, b in zip(g0, grads))
        kept = {"forward_ms_per_step": 1e3 * k_fwd / args.adj_steps,
                "backward_ms_per_step": 1e3 * k_bwd / args.adj_steps,
                "backward_over_forward_plain": k_bwd / t_plain,
                "peak_torch_allocated_bytes": int(torch.cuda.max_memory_allocated(dev)),
                "max_rel_diff_vs_checkpointed_gradient": agree,
                "how": "rollout(every = 0): the forward steps with the saving step kernel and keeps each "
                       "step's input and stage states; the backward runs the adjoint kernels only; "
                       "median of 3 timed rollouts"}
        del runs0, g0
    run.check()
    # device time of one backward step's two launches in a tight loop: the
    # saving step kernel and the adjoint kernel on fixed buffers
    sbuf = run.saved_buffer()
    st0 = {k: v.clone() for k, v in base.items()}
    ybar = {k: torch.ones_like(v) for k, v in base.items()}
    for _ in range(2):
        run.step_saving(st0, sbuf, eddy0, hs0)
        run.vjp(st0, ybar, eddy0, hs0, saved=sbuf)
    n_k = 10
    t_save = t_adj = 0.0
    for _ in range(n_k):
        a0, a1, a2, a3 = ev(), ev(), ev(), ev()
        run._load(st0, eddy0, hs0)
        a0.record()
        run.plan.advance_saving(DT, sbuf)
        a1.record()
        bars = {k: ybar[k].clone() for k in ybar}
        bars["eddy"] = torch.zeros_like(eddy0)
        bars["heating_scale"] = torch.zeros_like(hs0)
        run._load(st0, eddy0, hs0)
        a2.record()
        run.plan.adjoint([bars], DT, saved=sbuf)
        a3.record()
        a3.synchronize()
        t_save += a0.elapsed_time(a1) / 1e3
        t_adj += a2.elapsed_time(a3) / 1e3
    t_save /= n_k
    t_adj /= n_k
    clk = clocks.stop()
    del sbuf

    # finite differences: directions on one column each, eps = 1e-7 relative,
    # over one step and over the whole rollout; no direction is filtered out,
    # so directions that cross a limiter kink inside the rollout count as
    # they come
    def fd_errors(n_steps, grads_n):
        def per_column_J(state, ed, h):
            st = {k: v.clone() for k, v in state.items()}
            for _ in range(n_steps):
                st = run.step(st, ed, h)
            nd = st["ndensity_s"]
            return w * (torch.log(nd[0, lvl]) - torch.log(nd[2, lvl]))
        return _fd_errors(per_column_J, grads_n)

    def _fd_errors(per_column_J, grads):
        errs = []
        for trial in range(fd_directions):
            col = int(torch.randint(0, n_cols, (1,), generator=gen, device=dev))
            d = {}
            for k in names:
                dd = torch.zeros_like(base[k])
                dd[..., col] = torch.randn(dd[..., col].shape, generator=gen, device=dev, dtype=torch.float64)
                d[k] = dd
            de = torch.zeros_like(eddy0)
            de[..., col] = torch.randn(de[..., col].shape, generator=gen, device=dev, dtype=torch.float64)
            dh = torch.zeros_like(hs0)
            dh[col] = 1.0
            st = {k: base[k].abs() * eps for k in names}

            def point(sg):
                s2 = {k: base[k] + sg * d[k] * st[k] if k in d else base[k] for k in base}
                return s2, eddy0 + sg * de * eddy0.abs() * eps, hs0 + sg * dh * hs0.abs() * eps
            jp = per_column_J(*point(1.0))[col]
            jm = per_column_J(*point(-1.0))[col]
            fd = float(jp - jm) / 2.0
            ana = sum(float((g * d[k] * st[k]).sum()) for g, k in zip(grads[:5], names))
            ana += float((grads[5] * de * eddy0.abs() * eps).sum()) + float((grads[6] * dh * hs0.abs() * eps).sum())
            floor = 8 * 2.2e-16 * abs(float(jp))
            errs.append(max(abs(fd - ana) - floor, 0.0) / max(abs(fd), abs(ana), 1e-300))
        return np.array(errs)

    eps = 1e-7
    if fd_directions > 0:
        grads1 = grads_once(1)[0]
        errs1 = fd_errors(1, grads1)
        errs = fd_errors(args.adj_steps, grads)
    else:
        errs1 = errs = np.zeros(0)
    run.close()
    ctx.close()
    if rank == 0:
        n = args.adj_steps
        out = {"metric": "adjoint / forward cost per step, 2.5 deg rollout (10,368 columns x 50 alts)",
               "value": (t_bwd / n) / (t_plain / n), "unit": "ratio", "higher_is_better": False,
               "n_gpus": 1, "steps": n, "dtype": "f64", "data": "synthetic (seeded)",
               "config": {"workload": f"globe {args.adj_deg} deg, {n_cols} columns x {args.n_alts} alts, "
                                      f"Rusanov RK4, dt 2 s, {n} steps, checkpoint every {args.adj_every}",
                          "objective": "sum_c w_c log(n_O / n_N2) at 400 km, w_c ~ U[0,1]",
                          "wrt": "initial NDensityS, Temperature, Velocity, VerticalVelocity, Rho, "
                                 "KappaEddyDiffusion, per-column heating factor"},
               "forward_plain_ms_per_step": 1e3 * t_plain / n,
               "forward_checkpointed_ms_per_step": 1e3 * t_fwd / n,
               "backward_ms_per_step": 1e3 * t_bwd / n,
               "backward_device_ms_per_step": {"saving_step": 1e3 * t_save, "adjoint_kernel": 1e3 * t_adj,
                                               "how": "the two launches of a backward step on fixed buffers, "
                                                      "CUDA events around each, mean of 10"},
               "timing": "median of 3 timed rollouts",
               "clocks": clk,
               "stages_kept": kept,
               "backward_includes": "segment recompute (the step kernel saving its stage states; the last "
                                    "segment's were kept by the forward) + one adjoint kernel per step "
                                    "reading them",
               "objective_value": Jv,
               "peak_memory": {"torch_allocated_bytes": int(peak_torch),
                               "device_used_delta_bytes": int(free0 - free1)},
               "fd_check": {
                   "one_step": {"directions": int(len(errs1)), "within_1e-6": int((errs1 < 1e-6).sum()),
                                "median_rel_err": float(np.median(errs1)) if len(errs1) else None,
                                "max_rel_err": float(errs1.max()) if len(errs1) else None},
                   "rollout": {"steps": n, "directions": int(len(errs)), "within_1e-6": int((errs < 1e-6).sum()),
                               "median_rel_err": float(np.median(errs)) if len(errs) else None,
                               "max_rel_err": float(errs.max()) if len(errs) else None},
                   "eps_relative": eps,
                   "how": "central differences of the per-column objective, directions on one column "
                          "each, no direction filtered out, rounding floor of a few ulps of J "
                          "subtracted; the limiter's kinks are dense (a 1e-7 perturbation of one "
                          "column flips branches within a few steps), so rollout differences mix "
                          "branches; the branch-exact check is tests/test_gpu_adjoint.py"}}
        return out
    return None


# ---------------------------------------------------------------- ensemble
def tile_member(m, n: int):
    """The member's columns repeated to n columns (per-column arrays indexed
    modulo the generated count; the shared grid is kept)."""
    import dataclasses
    idx = np.arange(n) % m.n_cols
    kw = {}
    for f in dataclasses.fields(m):
        v = getattr(m, f.name)
        if isinstance(v, np.ndarray) and f.name not in ("altitude", "gravity", "dalt_c", "inv_r"):
            v = np.ascontiguousarray(v[..., idx])
        kw[f.name] = v
    kw["n_cols"] = n
    return type(m)(**kw)


def run_ensemble(args):
    """Uneven ensemble in one launch: members with resolutions drawn from
    {5x5, 2.5x2.5, 1x2} degrees and nAlts from {50, 75, 100}, each member's
    Tinf shifted by N(0, 100 K) and its heating scaled lognormally (sigma
    0.3), packed ragged into one plan (per-member offsets) and advanced in
    graph-captured launches; compared with looping the plain per-call drop-in
    over the members."""
    import torch

    from gitm_b200 import abi, synthetic
    from gitm_b200 import vertical as V

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    rng = np.random.default_rng(1000 + rank)
    res = [(5.0, 5.0), (2.5, 2.5), (1.0, 2.0)]
    members = []
    for k in range(args.ens_members):
        dlat, dlon = res[rng.integers(0, 3)]
        na = int(rng.choice([50, 75, 100]))
        n = int(round(180.0 / dlat)) * int(round(360.0 / dlon))
        # a block of up to 2,592 generated columns tiled to the member's size
        # (columns are independent; repeats change no cost)
        m = synthetic.make_member(min(n, 2592), n_alts=na, seed=10_000 * rank + k,
                                  tinf_shift=float(rng.normal(0.0, 100.0)), with_heating=True)
        m = tile_member(m, n)
        m.heating_scale = m.heating_scale * float(np.exp(rng.normal(0.0, 0.3)))
        members.append(m)
    n_cols = sum(m.n_cols for m in members)
    col_steps_per_step = n_cols
    ctx = V.VerticalContext(abi.default_params(), device=local)
    dms = [V.device_member(m, device=dev) for m in members]
    names = ("ndensity_s", "idensity_s", "rho", "temperature", "velocity", "vert_vel")
    snap = [{k: d.tensors[k].clone() for k in names} for d in dms]

    def restore():
        for d, sn in zip(dms, snap):
            for k in names:
                d.tensors[k].copy_(sn[k])

    # plain drop-in: one gitm_vert_advance_native call per member per step
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.ens_plain_steps):
        for d in dms:
            V.advance_vertical_all(ctx, [d], DT, 1)
    torch.cuda.synchronize()
    t_plain = (time.perf_counter() - t0) / args.ens_plain_steps
    restore()
    plan = V.Plan(ctx, dms)
    cfg = plan.autotune(DT, 2)
    restore()
    chunk = min(args.ens_steps, CHUNK)
    graph = torch.cuda.CUDAGraph()
    cap = torch.cuda.Stream(dev)
    cap.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(cap):
        with torch.cuda.graph(graph, stream=cap):
            plan.advance(DT, chunk, stream=cap)
    torch.cuda.synchronize()
    n_rep = -(-args.ens_steps // chunk)
    clocks = ClockSampler(local)
    clocks.start()
    el = 0.0
    for _ in range(n_rep):
        restore()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(cap):
            e0.record(cap)
            graph.replay()
            e1.record(cap)
        e1.synchronize()
        el += e0.elapsed_time(e1) / 1e3
    clk = clocks.stop()
    st, nbad = plan.status(clear=True)
    steps = n_rep * chunk
    launches = plan.launch_count(chunk) * n_rep
    plan.close()
    ctx.close()
    if rank == 0:
        na_hist = {str(a): sum(1 for m in members if m.n_alts == a) for a in (50, 75, 100)}
        out = {"metric": "column-steps/s, uneven ensemble in one launch", "value": col_steps_per_step * steps / el,
               "unit": "column-steps/s", "n_gpus": 1, "steps": steps, "warmup": 4,
               "ms_per_step": 1e3 * el / steps, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
               "config": {"workload": f"{len(members)} members, {n_cols} columns, resolutions 5x5 / 2.5x2.5 / "
                                      "1x2 deg, nAlts 50 / 75 / 100, Tinf shift N(0,100 K), heating x "
                                      "lognormal(0.3), Rusanov RK4, dt 2 s",
                          "members_by_nalts": na_hist, "columns": n_cols,
                          "launch": {"threads": cfg.threads, "steps_per_launch": cfg.steps_per_launch,
                                     "ctas_per_sm": cfg.ctas_per_sm, "graph": True, "graph_steps": chunk,
                                     "state_restored_every": chunk}},
               "clocks": clk, "gpu_launches": launches, "status": {"or": st, "bad_columns": nbad},
               "plain_loop": {"value": col_steps_per_step / t_plain, "unit": "column-steps/s",
                              "ms_per_step": 1e3 * t_plain,
                              "how": "gitm_vert_advance_native per member per step (plan built each call), "
                                     "wall clock"}}
        out["batched_over_plain"] = out["value"] / out["plain_loop"]["value"]
        return out
    return None


def measured_hbm_peak() -> float:
    """The measured HBM copy bandwidth (GB/s) of this pool's B200s, else the
    earlier pool measurement of 6.65 TB/s."""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except Exception:
        return 6650.0


def hz_bytes_per_block(n_lons: int, n_lats: int, n_alts: int) -> int:
    """DRAM bytes of one block per advance_horizontal, counted from above:
    every block array the step reads, once, whole (the state's 27 fields:
    Rho, Temperature, Velocity, VerticalVelocity, the six NDensityS,
    IDensityS; Gamma, two IVelocity components, IVelocityPar,
    RadialDistance and its inverse, the six lon / lat distances; two
    components of cMax_GDB with its one ghost cell), and the interior cells
    it writes (21 fields and HorizontalTempSource)."""
    whole = (n_lons + 4) * (n_lats + 4) * (n_alts + 4)
    cmax = (n_lons + 2) * (n_lats + 2) * (n_alts + 2)
    interior = n_lons * n_lats * n_alts
    read = (2 + 3 + 6 + 6 + 10) + (1 + 2 + 3 + 2 + 6)
    written = 2 + 3 + 6 + 6 + 3 + 1
    return 8 * (read * whole + 2 * cmax + written * interior)


def run_horizontal(args):
    """advance_horizontal (gitm_hz_advance) on a globe of 9 x 9 blocks at
    hz_deg: one launch per step over every (block, altitude) plane, state
    resident in HBM; cell-steps/s = interior cells x steps / device time.
    CPU baseline: the oracle on the host cores on a sample of the blocks."""
    import torch

    from gitm_b200 import abi
    from gitm_b200 import horizontal as H
    from gitm_b200 import vertical as V

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    nl = nt = 9
    nbl = int(round(360.0 / args.hz_deg)) // nl
    nbt = int(round(180.0 / args.hz_deg)) // nt
    blocks = H.synthetic_blocks(nl, nt, args.n_alts, nbl, nbt, seed=rank)
    cells = nl * nt * args.n_alts * blocks.n_blocks
    p = abi.default_hz_params()
    ctx = V.VerticalContext(abi.default_params(), device=local)
    d = blocks.to_device(torch.device("cuda", local))
    # the synthetic globe has no polar filter: at 1 deg the cells next to the
    # poles are ~1 km wide in longitude and a 2 s step exceeds their CFL
    # limit, so the state goes back to the initial one every `chunk` steps
    # (outside the timed region)
    snap = {k: d.arrays[k].clone() for k in H.OUTPUTS}

    def restore():
        for k in H.OUTPUTS:
            d.arrays[k].copy_(snap[k])
    chunk = 4
    for _ in range(max(args.warmup, 3)):
        H.advance_horizontal(ctx, d, DT, p)
    restore()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    stream = torch.cuda.current_stream()
    from gitm_b200._lib import lib
    import ctypes as C
    b = d.batch()
    x = H.exchange_batch(d)
    sp = C.c_void_p(stream.cuda_stream)

    def timed(with_exchange: bool) -> float:
        el = 0.0
        for _ in range(n_chunks):
            restore()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(chunk):
                # advance_horizontal_all (advance_horizontal.f90:8-49): exchange, advance, exchange
                if with_exchange and lib().gitm_hz_exchange(ctx.handle, C.byref(x), sp):
                    raise RuntimeError(ctx.last_error())
                if lib().gitm_hz_advance(ctx.handle, C.byref(p), C.byref(b), DT, sp):
                    raise RuntimeError(ctx.last_error())
                if with_exchange and lib().gitm_hz_exchange(ctx.handle, C.byref(x), sp):
                    raise RuntimeError(ctx.last_error())
            e1.record(stream)
            e1.synchronize()
            el += e0.elapsed_time(e1) / 1e3
        return el

    n_chunks = max(1, -(-args.hz_steps // chunk))
    el = timed(True)
    word, nbad = H.hz_status(ctx, clear=True)
    el_adv = timed(False)
    args.hz_steps = n_chunks * chunk
    clk = clocks.stop()
    w2, n2 = H.hz_status(ctx, clear=True)
    word, nbad = word | w2, max(nbad, n2)
    ctx.close()
    cb = None
    if rank == 0 and args.cpu_seconds > 0:
        from oracle import oracle
        threads = os.cpu_count() or 1
        nsample = min(blocks.n_blocks, max(threads, 64))
        sample = H.HzBlocks(nl, nt, args.n_alts, nsample,
                            {k: np.ascontiguousarray(v[:nsample]) for k, v in blocks.arrays.items()})
        t0 = time.perf_counter()
        oracle.hz_advance(sample, p, DT, nthreads=threads)
        ec = time.perf_counter() - t0
        cb = {"value": nl * nt * args.n_alts * nsample / ec, "unit": "cell-steps/s", "cores": threads,
              "kind": "port", "sample": f"{nsample} of {blocks.n_blocks} blocks x 1 step, C++ oracle -O3, "
                                        f"{threads} threads, {ec:.1f} s"}
    if rank == 0:
        per_step = el / args.hz_steps
        per_adv = el_adv / args.hz_steps  # the dominant kernel, alone
        bytes_step = hz_bytes_per_block(nl, nt, args.n_alts) * blocks.n_blocks
        peak = measured_hbm_peak()
        out = {"metric": f"cell-steps/s, horizontal step (exchange, advance_horizontal, exchange), "
                         f"{args.hz_deg:g} deg globe of 9x9 blocks",
               "value": cells / per_step, "unit": "cell-steps/s", "n_gpus": 1, "steps": args.hz_steps,
               "warmup": max(args.warmup, 3), "ms_per_step": 1e3 * per_step, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
               "config": {"workload": f"{blocks.n_blocks} blocks of {nl}x{nt} cells, {args.n_alts} alts, "
                                      f"advance_horizontal RK4, dt 2 s, improved ion advection",
                          "l2": "state larger than L2 (no flush needed)", "launch": "one CTA per (block, altitude) "
                          "plane; per step gitm_hz_exchange, gitm_hz_advance, gitm_hz_exchange",
                          "state_restored_every": 4},
               "clocks": clk, "gpu_launches": 3 * args.hz_steps, "status": {"or": word, "bad_blocks": nbad},
               "advance_only": {"value": cells / (el_adv / args.hz_steps), "unit": "cell-steps/s",
                                "ms_per_step": 1e3 * el_adv / args.hz_steps,
                                "how": "gitm_hz_advance alone, one launch per step"},
               "roofline_hbm": {"bound": "hbm", "kernel": "hz_step_kernel", "achieved": bytes_step / per_adv / 1e9,
                                "peak": peak, "unit": "GB/s", "frac": bytes_step / per_adv / 1e9 / peak,
                                "bytes_per_step": bytes_step,
                                "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"},
               "cpu_baseline": cb}
        print(json.dumps(out))


def main():
    args = parse()
    if args.horizontal:
        run_horizontal(args)
        return
    if args.ensemble:
        out = run_ensemble(args)
        if out:
            print(json.dumps(out))
        return
    if args.adjoint:
        out = run_adjoint(args)
        if out:
            print(json.dumps(out))
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
