#!/usr/bin/env python3
"""Throughput of the pyro_cmc Monte Carlo hot path on B200, in spin-updates/s.

Workload (the one line of output): the L=64 field-cool anneal
(4,194,304 spins, J1=1, J2=0.1, J3=0.05, B=(0,0,0.5), FP32 spins, FP64
accumulators). One step = one sampling temperature step of that anneal at
T=0.5: 32 Metropolis+overrelaxation sweeps, an S(q) sample of all nine
correlators after every 16 sweeps, one energy sample. A spin-update is one
Metropolis proposal at one site (each sweep also overrelaxes every site), so a
step is 32 * N spin-updates. Inputs are synthetic (uniform on S^2, device
Philox). The lattice (67 MB) is smaller than L2 (126 MB), so a 256 MiB buffer
is written between timed steps (outside the per-step CUDA events) and every
step starts with a cold L2.

  value   device-timed steps, spins resident in HBM (CUDA events on the
          system's stream, max over ranks)
  e2e     the same steps through the host-buffer C-ABI call pc_step_host3:
          pinned-host spins (x, y, z float32) in, spins and energy out, copies
          inside the timing; the float4 call pc_step_host beside it
  roofline  the fused colour-pass kernel: 32 B (float4 read + write) per
          updated site against the measured HBM copy bandwidth, with the
          survey's 64 B per spin-update and the L2 side beside it
  cpu_baseline  the reference's own src/MC.cpp sweep compiled unchanged
          (oracle/_ref; the oracle's FP64 restatement where it was not built)
          on one host core, on a bounded sample of the same lattice
Also reported: the batched parallel-tempering form (128 replicas, L in
{8,12,16,24} x 32 T; per-pass graphs and one persistent launch), the L=16
anneal step for one and for 32 seeds, and the gradient form (256 x L=8
energy + S^zz(q) loss, forward and backward with coupling gradients).

--gpus N runs N independent replicas of the workload, one per GPU (the path
has no exchange across GPUs): scaling "weak", value = all ranks' updates / the
slowest rank's time. --impl reference runs the CPU reference arm (the same
compiled reference code on all host threads) on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

METRIC = "spin-updates/s on 1 B200 (plain/batched/grad) at matched ⟨E⟩,C_v,S(q) vs CPU"
UNIT = "spin-updates/s"
WL = dict(L=64, J1=1.0, J2=0.1, J3=0.05, B=(0.0, 0.0, 0.5), T=0.5, n_sweep=32, ssf_every=16,
          corr=["xx", "yy", "zz", "xy", "xz", "yz", "yx", "zx", "zy"], schedule=1)
CONFIG = {"workload": "fieldcool L=64 sampling step (32 sweeps + 2 S(q) samples x 9 correlators + energy)",
          "L": 64, "n_spins": 16 * 64 ** 3, "J": [1.0, 0.1, 0.05], "B": [0.0, 0.0, 0.5], "T": 0.5,
          "n_sweep": 32, "ssf_every": 16, "n_corr": 9, "spins": "fp32", "accumulators": "fp64",
          "l2": "L2 flushed between timed steps (256 MiB buffer written outside the per-step events)", "parallelism": "replicas",
          "schedule": "fused: per colour class, each site's Metropolis move then its overrelaxation move with one "
                      "local field (pc_set_sweep_schedule 1); same moves per sweep as the reference's order"}


def max_over_ranks(x, dist=None, device="cuda"):
    """The maximum of a per-rank number over all ranks (the slowest rank's
    time); x itself without a process group."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, n_spins, sweeps, ms_max):
    """Spin-updates/s of the whole job: every rank updates its own replica
    (n_spins x sweeps per step), timed by the slowest rank."""
    return world * n_spins * sweeps / (ms_max * 1e-3)


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# Per-launch memory traffic of the fused colour pass at L = 64 from one ncu
# capture of the same kernel (bench.py --profile-case, a cold-L2 launch):
# DRAM bytes read + written, and L2 -> SM bytes. A profiler figure, reported
# with its source; the timed loop itself runs with the lattice L2-resident.
PROFILED_PASS = {"dram_bytes": 68618240.0, "l2_to_sm_bytes": 95.65e6, "lts_throughput_pct": 29.8,
                 "source": "ncu --set full of struct_pass_kernel, bench.py --profile-case (profiles/colour_pass_L64.md)"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"pyro_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # wait (at most 3 s) for the first sample, so the timed region is covered
        t0 = time.time()
        while time.time() - t0 < 3.0 and os.path.getsize(self.path) == 0 and self.proc.poll() is None:
            time.sleep(0.02)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------
def _ref_backend():
    """The reference's own src/MC.cpp compiled unchanged (oracle/_ref,
    kind "reference") where it was built, else the oracle's restatement of
    it (kind "port")."""
    from oracle import ref
    if ref.available():
        return "reference", lambda L, seed: ref.RefSystem(L, J1=WL["J1"], J2=WL["J2"], J3=WL["J3"], B=WL["B"],
                                                          seed=seed)
    import oracle
    return "port", lambda L, seed: oracle.System(L, J1=WL["J1"], J2=WL["J2"], J3=WL["J3"], B=WL["B"], seed=seed)


def _host_threads(gb_per_lattice):
    ncores = os.cpu_count() or 1
    mem_gb = 0.0
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                mem_gb = float(line.split()[1]) / 1e6
    except OSError:
        pass
    return max(1, min(ncores, int(mem_gb // gb_per_lattice) if mem_gb else ncores, 64))


def _cpu_sweeps(make, threads, sweeps, warmup):
    """`threads` independent L=64 lattices, one per host thread (the sweep
    runs outside the GIL), uniform random start; times `sweeps` sweeps of
    every lattice after `warmup`. Returns (spin-updates/s, seconds)."""
    import concurrent.futures as cf

    import numpy as np
    L, T = WL["L"], WL["T"]

    def build(k):
        m = make(L, 1 + k)
        rng = np.random.default_rng(k)
        S = rng.normal(size=(16 * L ** 3, 3))
        m.set_spins(S / np.linalg.norm(S, axis=1, keepdims=True))
        return m

    with cf.ThreadPoolExecutor(threads) as ex:
        systems = list(ex.map(build, range(threads)))
        list(ex.map(lambda m: m.sweep(T, warmup, 1), systems))
        t0 = time.perf_counter()
        list(ex.map(lambda m: m.sweep(T, sweeps, 1), systems))
        dt = time.perf_counter() - t0
    return threads * systems[0].N * sweeps / dt, dt


REF_CONFIG = {"workload": "reference sweep: sweep_local_Metropolis(T=0.5, n_overrelax=1) of src/MC.cpp on "
                          "independent L=64 lattices (4,194,304 spins each), one lattice per host thread; a step is "
                          "one sweep of every lattice",
              "L": 64, "n_spins": 16 * 64 ** 3, "J": [1.0, 0.1, 0.05], "B": [0.0, 0.0, 0.5], "T": 0.5,
              "n_sweep": 1, "ssf": "none", "energy": "none", "spins": "fp64", "move_order": "reference (sequential)",
              "parallelism": "independent lattices, one per thread"}


def run_reference(args, rank):
    """CPU reference arm: the reference's Monte Carlo sweep on all host cores,
    one independent L=64 lattice per thread; each step is one sweep of every
    lattice (the S(q) and energy samples of the GPU step are not run: the
    per-update rate is compared)."""
    if rank != 0:
        return
    kind, make = _ref_backend()
    threads = _host_threads(4.0)
    rate, dt = _cpu_sweeps(make, threads, args.steps, args.warmup)
    sample = (f"{args.steps} timed sweeps (after {args.warmup} warm-up) of {threads} independent L=64 lattices "
              f"(one per thread); Metropolis + overrelaxation, no S(q), no energy")
    line = {"metric": METRIC, "value": rate, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(REF_CONFIG, threads=threads, code=("src/MC.cpp compiled unchanged (oracle/_ref)"
                                                              if kind == "reference" else "oracle restatement")),
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_profile_case(args):
    """One step of the workload (32 fused sweeps, two 9-correlator S(q)
    samples, one energy) on a fresh system with a fixed tile: the launch
    sequence is random_spins, then per sweep one struct_pass launch per colour
    class (16), the S(q) kernels after sweeps 16 and 32, the energy kernels."""
    import torch

    import pyro_cmc_b200 as pc
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    s = pc.pyrochlore_system(WL["L"], J1=WL["J1"], J2=WL["J2"], J3=WL["J3"], B=WL["B"], seed=1000,
                             schedule=WL["schedule"])
    s.set_stream(stream.cuda_stream)
    s.set_tile(args.tile[0], args.tile[1])
    s.set_load_variant(args.tile[2])
    s.random_spins(17)
    s.ssf_configure(WL["corr"], 1)
    l0 = s.launch_count()
    for _ in range(WL["n_sweep"] // WL["ssf_every"]):
        s.sweep(WL["T"], WL["ssf_every"], 1, count=False)
        s.ssf_sample([0])
    e, _ = s.energy()
    torch.cuda.synchronize()
    print(f"profile case: L={WL['L']} tile={args.tile} launches={s.launch_count() - l0} e={e[0]:.6f}", flush=True)
    del s


def run_profile_grad(args):
    """One forward and backward of the gradient form (256 x L=8: energy with
    its spin gradient, S^zz(q) with its adjoint) after one warm-up, for ncu
    captures of the gradient kernels."""
    import torch

    import pyro_cmc_b200 as pc
    from pyro_cmc_b200 import autograd as ag
    torch.cuda.set_device(0)
    B = 256
    g = pc.pyrochlore_system(8, n_replicas=B, J1=1.0, J2=0.1, J3=-0.05, B=(0.2, 0, 0), seed=3)
    g.ssf_configure(["zz"], 0, [])
    g.random_spins(11)
    spins = ag.spins_tensor(g).clone().requires_grad_(True)
    w = torch.rand((B, 1, 512), device="cuda", dtype=torch.float64)
    for _ in range(2):
        e = ag.energy(g, spins)
        S = ag.ssf(g, spins)
        ((w * S[..., 0] ** 2).sum() * 1e-8 + e.sum()).backward()
    torch.cuda.synchronize()
    print(f"profile grad: 256 x L=8, launches={g.launch_count()}", flush=True)


def run_profile_batched(args):
    """The batched tempering form (128 replicas, L in {8,12,16,24} x 32 T,
    exchange every 10 sweeps, S(q) every 16) with a fixed tile and no
    autotuning: 4 rounds of 10 sweeps, for ncu launch lists."""
    import numpy as np
    import torch

    import pyro_cmc_b200 as pc
    torch.cuda.set_device(0)
    Ls = [8] * 32 + [12] * 32 + [16] * 32 + [24] * 32
    T = np.concatenate([np.geomspace(2.0, 0.02, 32)] * 4)
    b = pc.pyrochlore_system(Ls, J1=1.0, J2=0.0, J3=0.02, B=(0, 0, 0.1), seed=7, schedule=WL["schedule"])
    b.set_tile(args.tile[0], args.tile[1])
    b.set_load_variant(args.tile[2])
    b.random_spins(5)
    b.pt_configure(T)
    b.ssf_configure(["xx", "yy", "zz"], len(Ls), sorted(Ls))
    if args.persistent:
        b.set_pt_persistent(True)
    b.pt_run(4, 10, 16)
    torch.cuda.synchronize()
    print(f"profile batched: 128 replicas, tile={args.tile}, persistent={args.persistent}, "
          f"launches={b.launch_count()}", flush=True)


def run_profile_energy(args):
    """Three energy evaluations of the L = 64 field-cool lattice (uniform
    random spins), for ncu captures of the per-cell energy kernel."""
    import torch

    import pyro_cmc_b200 as pc
    torch.cuda.set_device(0)
    s = pc.pyrochlore_system(WL["L"], J1=WL["J1"], J2=WL["J2"], J3=WL["J3"], B=WL["B"], seed=1)
    s.random_spins(1)
    for _ in range(3):
        s.energy()
    torch.cuda.synchronize()
    print(f"profile energy: L={WL['L']}, launches={s.launch_count()}", flush=True)


def cpu_baseline_one_core():
    kind, make = _ref_backend()
    rate, _ = _cpu_sweeps(make, 1, 4, 1)
    return {"value": rate, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": "4 sweeps of one L=64 lattice (4,194,304 spins) after one warm-up sweep, single thread, "
                      "Metropolis + overrelaxation (no S(q)), "
                      + ("the reference's src/MC.cpp compiled unchanged" if kind == "reference"
                         else "the oracle's restatement")}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-extras", action="store_true", help="skip the batched and gradient forms")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--profile-case", action="store_true",
                    help="run one step of the workload with a fixed tile and no autotuning or warm-up, for ncu "
                         "captures (prints a launch summary, no JSON line)")
    ap.add_argument("--profile-batched", action="store_true",
                    help="4 tempering rounds of the batched form with a fixed tile, for ncu captures (no JSON line)")
    ap.add_argument("--persistent", action="store_true",
                    help="with --profile-batched: the rounds in one persistent launch")
    ap.add_argument("--profile-energy", action="store_true",
                    help="three energy evaluations of the L = 64 lattice, for ncu captures (no JSON line)")
    ap.add_argument("--profile-grad", action="store_true",
                    help="one warm-up and one forward + backward of the gradient form, for ncu captures (no JSON line)")
    ap.add_argument("--tile", type=int, nargs=3, default=[128, 7, 0], metavar=("THREADS", "CTAS", "VARIANT"),
                    help="tile for --profile-case")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    rank = env_int("RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    local = env_int("LOCAL_RANK", 0)

    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.profile_case:
        run_profile_case(args)
        return
    if args.profile_grad:
        run_profile_grad(args)
        return
    if args.profile_batched:
        run_profile_batched(args)
        return
    if args.profile_energy:
        run_profile_energy(args)
        return

    import numpy as np
    import torch

    import pyro_cmc_b200 as pc

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    s = pc.pyrochlore_system(WL["L"], J1=WL["J1"], J2=WL["J2"], J3=WL["J3"], B=WL["B"], seed=1000 + rank,
                             schedule=WL["schedule"])
    s.set_stream(stream.cuda_stream)
    s.random_spins(17 + rank)
    tile = s.autotune()
    s.ssf_configure(WL["corr"], 1)
    N = s.N()
    T = WL["T"]

    sweep_ev = []  # (start, end) CUDA events around the graph-launched sweeps of the timed steps

    def device_step(record=False):
        for _ in range(WL["n_sweep"] // WL["ssf_every"]):
            if record:
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
            s.sweep(T, WL["ssf_every"], 1, count=False)
            if record:
                b.record(stream)
                sweep_ev.append((a, b))
            s.ssf_sample([0])
        s.energy()

    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]

    def timed_steps(record=False):
        """K steps, each bracketed by CUDA events on the system's stream, L2
        flushed before each; returns the mean step time in ms."""
        for i in range(args.steps):
            flush_buf.zero_()
            starts[i].record(stream)
            device_step(record=record)
            ends[i].record(stream)
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in zip(starts, ends)) / args.steps

    for _ in range(args.warmup):
        device_step()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = s.launch_count()
    ms = timed_steps(record=True)
    launches = s.launch_count() - l0
    # mean colour-pass launch duration inside the timed steps: the sweeps'
    # event spans (graphs of 16 sweeps, overlapped launches) over their launches
    passes = args.steps * WL["n_sweep"] * s.colours()[0]
    t_pass = sum(a.elapsed_time(b) for a, b in sweep_ev) / passes
    barrier()
    clk = clocks.stop()
    ms_max = max_over_ranks(ms, dist)
    value = whole_job_rate(world, N, WL["n_sweep"], ms_max)

    # the same steps in the reference's move order (Metropolis pass, then the
    # overrelaxation pass), for comparison
    s.set_sweep_schedule(0)
    for _ in range(2):
        device_step()
    torch.cuda.synchronize()
    ms_ref_order = max_over_ranks(timed_steps(), dist)
    s.set_sweep_schedule(WL["schedule"])
    device_step()

    # for comparison: events around every single launch (no graph, no overlap)
    s.set_kernel_timing(True)
    device_step()
    t_met_isolated, _ = s.kernel_times()
    s.set_kernel_timing(False)

    # end to end through host buffers: the packed (x, y, z) call, and the
    # float4 call beside it
    def time_e2e(step, cols):
        S_in = torch.empty((N, cols), dtype=torch.float32, pin_memory=True).numpy()
        S_out = torch.empty((N, cols), dtype=torch.float32, pin_memory=True).numpy()
        S_in[:] = s.spins_f4()[:, :cols]
        for _ in range(args.warmup):
            step(S_in, S_out, T, WL["n_sweep"], WL["ssf_every"], 0)
        barrier()
        tot = 0.0
        for _ in range(args.steps):
            flush_buf.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            step(S_in, S_out, T, WL["n_sweep"], WL["ssf_every"], 0)  # returns after the D2H copy
            tot += time.perf_counter() - t0
        return max_over_ranks(tot / args.steps, dist)

    e2e_s = time_e2e(s.step_host3, 3)
    e2e4_s = time_e2e(s.step_host, 4)
    e2e = {"value": world * N * WL["n_sweep"] / e2e_s, "unit": UNIT, "h2d_bytes_per_step": N * 12,
           "d2h_bytes_per_step": N * 12 + 8, "ms_per_step": e2e_s * 1e3,
           "call": "pc_step_host3 (pinned host spins as x, y, z float32 in and out)",
           "float4": {"value": world * N * WL["n_sweep"] / e2e4_s, "ms_per_step": e2e4_s * 1e3,
                      "h2d_bytes_per_step": N * 16, "d2h_bytes_per_step": N * 16 + 8,
                      "call": "pc_step_host (pinned host spins as float4 in and out)"}}

    peak, peak_kind = measured_peaks()
    alg_bytes = 32.0 * s.Nc()  # one colour pass: one sublattice, float4 read + write per site
    achieved = alg_bytes / (t_pass * 1e-3) / 1e9 if t_pass > 0 else None
    l2_bytes = PROFILED_PASS["l2_to_sm_bytes"]
    gather_bytes = 32 * 16.0 * s.Nc()  # per site: own float4 read + write and 30 neighbour float4 loads
    roofline = {"bound": "hbm", "kernel": "struct_pass_kernel (fused Metropolis + overrelaxation colour pass)",
                "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                "frac": achieved / peak if achieved else None,
                "frac_survey_64B": (64.0 * s.Nc() / (t_pass * 1e-3) / 1e9) / peak if t_pass > 0 else None,
                "traffic": PROFILED_PASS["dram_bytes"], "traffic_source": "profile: " + PROFILED_PASS["source"],
                "alg_bytes_per_launch": alg_bytes, "launch_ms": t_pass, "launch_ms_isolated": t_met_isolated,
                "l2": {"l2_to_sm_bytes_per_launch": l2_bytes, "source": "profile: " + PROFILED_PASS["source"],
                       "gather_request_bytes_per_launch": gather_bytes,
                       "l2_to_sm_gbs": l2_bytes / (t_pass * 1e-3) / 1e9 if t_pass > 0 else None,
                       "lts_throughput_pct_of_peak": PROFILED_PASS["lts_throughput_pct"]},
                "note": "achieved = 32 B x Nc sites per launch / mean launch duration: CUDA events around the "
                        "graph-launched sweeps of the timed steps over their colour-pass launches (inter-kernel "
                        "gaps included); launch_ms_isolated: events around single launches outside graphs. "
                        "frac_survey_64B counts 64 B per spin-update (Metropolis + overrelaxation read + write, "
                        "the survey's accounting) for the same launch. The lattice (67 MB) stays in L2 during "
                        "the timed loop; the neighbour gathers are L2 -> SM traffic (l2): the profiled bytes per launch "
                        "over this run's launch time, and the L2 throughput ncu reports for the launch as a share "
                        "of the L2's own peak"}

    extras = {}
    if not args.no_extras and rank == 0:
        extras = run_extras(pc, torch, np)

    if rank == 0:
        cpu = None if (args.no_cpu or world > 1) else cpu_baseline_one_core()
        CONFIG["tile"] = {"threads": tile[0], "ctas_per_sm": tile[1], "load_variant": tile[2],
                          "chosen_by": "pc_autotune"}
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": CONFIG,
                "e2e": e2e, "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu,
                "clocks": clk}
        line["value_reference_order"] = {"value": world * N * WL["n_sweep"] / (ms_ref_order * 1e-3), "unit": UNIT,
                                          "ms_per_step": ms_ref_order, "schedule": "pc_set_sweep_schedule 0"}
        line.update(extras)
        print(json.dumps(line), flush=True)
    del s
    if dist is not None:
        dist.destroy_process_group()


def run_extras(pc, torch, np):
    out = {}
    stream = torch.cuda.current_stream()  # the non-default stream main() set
    # batched parallel tempering: 128 replicas, L in {8,12,16,24} x 32 T in [0.02, 2]
    Ls = [8] * 32 + [12] * 32 + [16] * 32 + [24] * 32
    Tl = np.geomspace(2.0, 0.02, 32)
    T = np.concatenate([Tl] * 4)
    b = pc.pyrochlore_system(Ls, J1=1.0, J2=0.0, J3=0.02, B=(0, 0, 0.1), seed=7, schedule=WL["schedule"])
    b.set_stream(stream.cuda_stream)
    b.random_spins(5)
    btile = b.autotune()
    b.pt_configure(T)
    b.ssf_configure(["xx", "yy", "zz"], len(Ls), sorted(Ls))
    b.pt_run(8, 10, 16)  # warm-up and graph capture (80 sweeps)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    rounds = 40
    e0.record(stream)
    b.pt_run(rounds, 10, 16)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    n_tot = sum(16 * L ** 3 for L in Ls)
    batched = n_tot * rounds * 10 / (ms * 1e-3)
    att, acc = b.pt_exchange_stats()
    # the same rounds in one persistent cooperative launch per stretch of
    # sweeps between S(q) samples (pc_set_pt_persistent)
    b.set_pt_persistent(True)
    b.pt_run(2, 10, 16)
    torch.cuda.synchronize()
    l0 = b.launch_count()
    e0.record(stream)
    b.pt_run(rounds, 10, 16)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_p = e0.elapsed_time(e1)
    launches_p = b.launch_count() - l0
    del b
    # plain single small replica (L=8), the comparison point for batching
    p1 = pc.pyrochlore_system(8, J1=1.0, J2=0.0, J3=0.02, B=(0, 0, 0.1), seed=9, schedule=WL["schedule"])
    p1.set_stream(stream.cuda_stream)
    p1.random_spins(1)
    p1.sweep(0.5, 20, 1, count=False)
    torch.cuda.synchronize()
    e0.record(stream)
    p1.sweep(0.5, 200, 1, count=False)
    e1.record(stream)
    torch.cuda.synchronize()
    plain_small = p1.N() * 200 / (e0.elapsed_time(e1) * 1e-3)
    del p1
    out["batched"] = {"value": batched, "unit": UNIT,
                      "config": "parallel tempering, 128 replicas (L 8/12/16/24 x 32 T geometric in [0.02, 2]), "
                                "J=(1,0,0.02), B=(0,0,0.1), exchange every 10 sweeps, S(q) xx/yy/zz every 16 sweeps",
                      "ms_per_10_sweeps": ms / rounds, "tile": list(btile), "exchange_accept": float(acc.sum()) / max(1.0, float(att.sum())),
                      "persistent": {"value": n_tot * rounds * 10 / (ms_p * 1e-3), "ms_per_10_sweeps": ms_p / rounds,
                                     "kernel_launches_per_round": launches_p / rounds},
                      "plain_single_L8": plain_small, "batched_over_plain_L8": batched / plain_small}
    # plain single replica of the L=16 anneal: one sampling step = 16 sweeps +
    # one S(q) sample of the anneal's six correlators
    a = pc.pyrochlore_system(16, J1=1.0, J2=-0.1, J3=0.05, B=(0, 0, 0), seed=21, schedule=WL["schedule"])
    a.set_stream(stream.cuda_stream)
    a.random_spins(2)
    atile = a.autotune()
    a.ssf_configure(["xx", "yy", "zz", "xy", "xz", "yz"], 1)

    def a_step():
        a.sweep(0.5, 16, 1, count=False)
        a.ssf_sample([0])

    for _ in range(5):
        a_step()
    torch.cuda.synchronize()
    n_a = 50
    e0.record(stream)
    for _ in range(n_a):
        a_step()
    e1.record(stream)
    torch.cuda.synchronize()
    a_ms = e0.elapsed_time(e1) / n_a
    # the same anneal step for the K = 32 seeds its statistics need, batched
    # as replicas of one system
    K = 32
    a2 = pc.pyrochlore_system(16, n_replicas=K, J1=1.0, J2=-0.1, J3=0.05, B=(0, 0, 0), seed=22,
                              schedule=WL["schedule"])
    a2.set_stream(stream.cuda_stream)
    a2.random_spins(3)
    a2.autotune()
    a2.ssf_configure(["xx", "yy", "zz", "xy", "xz", "yz"], K)
    slots = np.arange(K, dtype=np.int32)

    def a2_step():
        a2.sweep(0.5, 16, 1, count=False)
        a2.ssf_sample(slots)

    for _ in range(3):
        a2_step()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(10):
        a2_step()
    e1.record(stream)
    torch.cuda.synchronize()
    a2_ms = e0.elapsed_time(e1) / 10
    del a2
    out["plain_L16_32_seeds"] = {"value": K * 16 * 16 ** 3 * 16 / (a2_ms * 1e-3), "unit": UNIT,
                                 "config": "the L=16 anneal step for 32 seeds batched as replicas of one system",
                                 "ms_per_step": a2_ms}
    out["plain_L16"] = {"value": a.N() * 16 / (a_ms * 1e-3), "unit": UNIT,
                        "config": "anneal L=16 (65,536 spins), J=(1,-0.1,0.05), B=0, T=0.5; step = 16 sweeps + "
                                  "one S(q) sample (xx,yy,zz,xy,xz,yz)",
                        "ms_per_step": a_ms, "tile": list(atile)}
    del a
    # gradient form (the gradient configuration): 256 x L=8 uniform random
    # configurations, J = (1, 0.1, -0.05), B = (0.2, 0, 0); objective = energy
    # (with its gradients in the spins, J1..J3 and B) + sum_q w(q) |S^zz(q) -
    # S_target(q)|^2, w ~ U[0, 1], S_target = S^zz of the spiral_byhand state
    # at a seeded random Q
    from pyro_cmc_b200 import autograd as ag
    from pyro_cmc_b200 import ssf_fit
    B = 256
    g = pc.pyrochlore_system(8, n_replicas=B, J1=1.0, J2=0.1, J3=-0.05, B=(0.2, 0, 0), seed=3)
    g.set_stream(stream.cuda_stream)
    g.ssf_configure(["zz"], 0, [])
    rng = np.random.default_rng(4)
    Q = rng.integers(0, 8, size=3)
    target = torch.as_tensor(ssf_fit.zz_target(g, Q), device="cuda")
    g.random_spins(11)
    spins = ag.spins_tensor(g).clone().requires_grad_(True)
    params = torch.tensor([1.0, 0.1, -0.05, 0.2, 0.0, 0.0], dtype=torch.float64, requires_grad=True)
    w = torch.as_tensor(rng.uniform(0, 1, 512), device="cuda")
    lam = 1.0 / float((w * target ** 2).sum())

    def fwd_bwd():
        spins.grad = None
        params.grad = None
        e = ag.energy(g, spins, params)
        loss = e.sum() + lam * ssf_fit.weighted_zz_loss(ag.ssf(g, spins), w, target).sum()
        loss.backward()
        return loss

    for _ in range(3):
        fwd_bwd()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(5):
        with torch.no_grad():
            e = ag.energy(g, spins, params)
            lam * ssf_fit.weighted_zz_loss(ag.ssf(g, spins), w, target).sum() + e.sum()
    e1.record(stream)
    torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1) / 5
    e0.record(stream)
    for _ in range(5):
        fwd_bwd()
    e1.record(stream)
    torch.cuda.synchronize()
    fb_ms = e0.elapsed_time(e1) / 5
    out["grad"] = {"value": B * g.N() / (fb_ms * 1e-3), "unit": "spins/s (energy + S^zz(q) loss, forward and backward)",
                   "config": "256 x L=8 (2,097,152 spins), J=(1,0.1,-0.05), B=(0.2,0,0); loss = e + "
                             "sum_q w(q)|S^zz(q) - S_target(q)|^2 / norm, w ~ U[0,1], S_target = S^zz of the "
                             "spiral_byhand state at seeded random Q; gradients in the spins, J1..J3 and B",
                   "forward_ms": fwd_ms, "forward_backward_ms": fb_ms,
                   "backward_over_forward": (fb_ms - fwd_ms) / fwd_ms}
    del g
    return out


if __name__ == "__main__":
    main()
