#!/usr/bin/env python
"""Benchmark of the hst RK3 / Crank-Nicolson substep on B200s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config c3]

One step is one RK3 time step (three substeps, hst_gpu_timestep, with the
CFL read-back the Fortran time loop does every step); the metric is
substeps per second of the whole job.  Default workload: the plain FP64
drop-in at 768x768 dealiased x 512 ("512^3": deck nx = 255, nz = 256,
ny = 512; ly = 2 pi, alfa0 = beta0 = 1, S = 1, Re = 5000, dt = 0.001,
exact_shift) from a seeded divergence-free field with
E(k) ~ k^4 exp(-2 (k/16)^2), energy 0.1.  The same line carries the
mixed-precision form on the same field (`mixed`), each form's error against
the oracle after the same substeps (`accuracy`), the end-to-end rate through
the C ABI with host buffers (`e2e`), the roofline of the top kernel and of
the whole substep, and the oracle timed on the host cores (`cpu_baseline`).
The fields (gigabytes) are far larger than L2, so no flush is needed.

N > 1 (one process per GPU under torch.distributed.run): independent
replicas of the single-field path, which does not shard (the reference's
pencil decomposition exists to spread one field over many GPUs; here one
B200 holds it); no collective inside a step.  value = all ranks' substeps /
the max over ranks of the device-timed region.

--impl reference: the reference's CPU path on the host cores.  The
reference (Fortran + MPI + FFTW) cannot be built in this image, so its
restatement in oracle/ is timed instead (all host threads), rank 0 only;
each of its steps is one substep of the same workload (a bounded sample:
a substep of the 768^2 x 512 field takes the host seconds).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PI = math.pi

from homogenenousshearturbulence_b200.workloads import ENSEMBLE, ENSEMBLE_COMMON, ENSEMBLE_K0, WORKLOADS  # noqa: E402

# the workloads this script times, with the substeps of the oracle run that
# gives the CPU baseline and the accuracy (about 10-30 s of host time on 16
# threads; one warm-up substep first); the 1536^2 x 512 field has no CPU leg:
# one oracle substep of it needs about 90 GB of host memory and minutes
CONFIGS = {k: dict(v, label="FP64 substep, " + v["label"]) for k, v in WORKLOADS.items()}
ORACLE_SUBSTEPS = {"c1": 60, "c2": 12, "c3": 3, "c5": 0}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def alg_bytes(deck, nxd, nzd, split, mixed=False, shift_split=False):
    """Compulsory HBM bytes per launch of each kernel and per substep.
    Ns = ny (2nz+1)(nx+1) spectral points per component, Nzx = ny nzd (nx+1).
    With the column stage split, `rhs` streams V, Q, old in and old, rhs out
    (15 Ns) and `column` reads rhs and writes V (5 Ns; 9 Ns with exact_shift,
    which re-reads and rewrites old); fused, `column` moves 16 Ns.  The
    substep figure is the four-pass model 16 (25 Ns + 18 Nzx).  Mixed
    precision: Z, Pp and Q are 8-byte complex64, V, old and rhs stay 16-byte
    complex128; the substep model becomes 16 13 Ns + 8 (12 Ns + 18 Nzx)."""
    nx, ny, nz = deck["nx"], deck["ny"], deck["nz"]
    Ns = ny * (2 * nz + 1) * (nx + 1)
    Nzx = ny * nzd * (nx + 1)
    b, t = 16.0, (8.0 if mixed else 16.0)
    k = {
        "zinv": b * 3 * Ns + t * 3 * Nzx,
        "xprod": t * (3 * Nzx + 6 * Nzx),
        "zfwd": t * (6 * Nzx + 6 * Ns),
        "rhs": b * 9 * Ns + t * 6 * Ns,
        "column": b * ((9 if deck.get("exact_shift") and not shift_split else 5) * Ns if split else 10 * Ns)
                  + (0 if split else t * 6 * Ns),
        # the exact_shift shift as a kernel of its own: rhs and old in and out
        "shift": b * 8 * Ns,
    }
    sub = b * 13 * Ns + t * (12 * Ns + 18 * Nzx)
    return k, sub, Ns, Nzx


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def seeded_field(cfg, y):
    from homogenenousshearturbulence_b200 import hst
    d = cfg["deck"]
    return hst.random_field(d["nx"], d["ny"], d["nz"], d["alfa0"], d["beta0"], d["ly"], y, seed=1, k0=cfg["k0"],
                            energy=0.1)


def run_ensemble(args, dev):
    """Every member in its own context and stream: the concurrent form queues
    one time step of each member in turn (hst_gpu_timesteps, no host wait)
    and times the whole ensemble between two events that all member streams
    are joined to; the sequential form advances the members one after
    another with the CFL read-back of every step, as 32 separate plain runs
    would.  Returns (concurrent, sequential) member-substeps/s and the
    per-member device bytes."""
    import torch
    from homogenenousshearturbulence_b200 import hst
    members = []
    for i, sz in enumerate(ENSEMBLE):
        deck = dict(ENSEMBLE_COMMON, **sz, precision=args.precision)
        s = hst.Solver(deck, device=dev)
        V0 = hst.random_field(deck["nx"], deck["ny"], deck["nz"], deck["alfa0"], deck["beta0"], deck["ly"], s.y,
                              seed=i + 1, k0=ENSEMBLE_K0, energy=0.1)
        s.time = 0.0
        s.set_velocity(V0)
        members.append(s)
    dt = ENSEMBLE_COMMON["deltat"]
    streams = [torch.cuda.ExternalStream(s.stream, device=torch.device("cuda", dev)) for s in members]
    main = torch.cuda.current_stream(dev)

    def concurrent(k):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(main)
        for st in streams:
            st.wait_event(e0)
        for _ in range(k):
            for s in members:
                s.timesteps(1, dt)
        for st in streams:
            ev = torch.cuda.Event()
            ev.record(st)
            main.wait_event(ev)
        e1.record(main)
        e1.synchronize()
        return e0.elapsed_time(e1)

    def sequential(k):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(main)
        for s, st in zip(members, streams):
            st.wait_event(e0)
            for _ in range(k):
                s.timestep(dt)
            ev = torch.cuda.Event()
            ev.record(st)
            main.wait_event(ev)
        e1.record(main)
        e1.synchronize()
        return e0.elapsed_time(e1)

    concurrent(max(3, args.warmup))
    torch.cuda.synchronize(dev)
    ms_c = concurrent(args.steps)
    ms_s = sequential(max(3, args.steps // 3))
    n = len(members)
    rate_c = 3 * n * args.steps / (ms_c / 1000.0)
    rate_s = 3 * n * max(3, args.steps // 3) / (ms_s / 1000.0)
    cfl_ok = all(math.isfinite(s.compute_cfl()) for s in members)
    for s in members:
        s.close()

    # the batched form: one ensemble context per member shape (24 and 8
    # members), each kernel of the substep covering all of its members in one
    # launch; the two contexts' streams run side by side
    groups = {}
    for i, sz in enumerate(ENSEMBLE):
        groups.setdefault(tuple(sorted(sz.items())), []).append(i)
    ens = []
    for key, idx in groups.items():
        deck = dict(ENSEMBLE_COMMON, **dict(key), precision=args.precision)
        e = hst.Solver(deck, device=dev, members=len(idx))
        e.time = 0.0
        for m, i in enumerate(idx):
            e.select(m)
            e.set_velocity(hst.random_field(deck["nx"], deck["ny"], deck["nz"], deck["alfa0"], deck["beta0"],
                                            deck["ly"], e.y, seed=i + 1, k0=ENSEMBLE_K0, energy=0.1))
        ens.append(e)
    estreams = [torch.cuda.ExternalStream(e.stream, device=torch.device("cuda", dev)) for e in ens]

    def batched(k):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(main)
        for st in estreams:
            st.wait_event(e0)
        for _ in range(k):
            for e in ens:
                e.timesteps(1, dt)
        for st in estreams:
            ev = torch.cuda.Event()
            ev.record(st)
            main.wait_event(ev)
        e1.record(main)
        e1.synchronize()
        return e0.elapsed_time(e1)

    batched(max(3, args.warmup))
    torch.cuda.synchronize(dev)
    ms_b = batched(args.steps)
    rate_b = 3 * n * args.steps / (ms_b / 1000.0)
    cfl_ok = cfl_ok and all(math.isfinite(e.compute_cfl()) for e in ens)
    for e in ens:
        e.close()
    return rate_b, rate_c, rate_s, ms_b, cfl_ok


def reduce_max(x, dist, device=None):
    """The maximum over ranks of a float (the device time of the timed
    region); x itself without a process group."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, units_per_rank, ms_max):
    """Units per second of the whole job: every rank's units over the
    slowest rank's time."""
    return world * units_per_rank / (ms_max / 1000.0)


def oracle_substeps(cfg, warmup, timed, V0=None):
    """The oracle (the reference's CPU path restated, all host threads) on
    the workload from its seeded field: `warmup` untimed substeps, then
    `timed` timed ones (substep i of a time step is i mod 3).  Returns
    (substeps/s, threads, the velocity after all of them, the time)."""
    import oracle
    d = dict(cfg["deck"])
    o = oracle.Sim(oracle.params_from_deck(d))
    if V0 is None:
        V0 = seeded_field(cfg, o.y())
    for c in range(3):
        o.field(c)[...] = V0[c]
        o.fill_ghosts(c)
    o.time = 0.0
    o.deltat = d["deltat"]
    for k in range(warmup):
        o.substep(k % 3)
    t0 = time.perf_counter()
    for k in range(warmup, warmup + timed):
        o.substep(k % 3)
    el = time.perf_counter() - t0
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    V = np.stack([o.field(c).copy() for c in range(3)])
    return (timed / el if timed else float("nan")), threads, V, o.time


def cpu_oracle_rate(cfg, steps, budget_s=60.0, warmup=1):
    """Substeps/s of the oracle on the workload: one warm-up substep, then
    timed substeps within the budget (at most 3 steps); returns (substeps/s,
    substeps timed, threads, warm-up substeps)."""
    import oracle
    d = dict(cfg["deck"])
    o = oracle.Sim(oracle.params_from_deck(d))
    V0 = seeded_field(cfg, o.y())
    for c in range(3):
        o.field(c)[...] = V0[c]
        o.fill_ghosts(c)
    o.deltat = d["deltat"]
    t0 = time.perf_counter()
    o.substep(0)
    first = time.perf_counter() - t0
    n = max(1, min(3 * steps, int(budget_s / max(first, 1e-6))))
    t0 = time.perf_counter()
    for k in range(1, 1 + n):
        o.substep(k % 3)
    el = time.perf_counter() - t0
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return n / el, n, threads, 1


def ensemble_main(args):
    """--config c4: the batched ensemble on one GPU (rank 0 of each process
    runs its own ensemble; the reference arm times the oracle on the first
    small member, the reference having no batched form)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    unit = "substeps/s"
    label = ("ensemble of 32 independent realisations in one GPU: 24 x 192^2 x 128 (nx=63, nz=64, ny=128) + "
             "8 x 384^2 x 192 (nx=95, nz=96, ny=192), Re 1500, dt 0.004, seeds 1..32")
    if args.impl == "reference":
        if rank != 0:
            return 0
        cfg = dict(deck=dict(ENSEMBLE_COMMON, **ENSEMBLE[0]), k0=ENSEMBLE_K0)
        rate, n, threads, w = cpu_oracle_rate(cfg, args.steps, budget_s=60.0, warmup=args.warmup)
        # the members one after another: a substep of every member takes
        # 24 small and 8 large member-substeps
        small = rate
        big_cfg = dict(deck=dict(ENSEMBLE_COMMON, **ENSEMBLE[-1]), k0=ENSEMBLE_K0)
        rate_b, nb, _, _ = cpu_oracle_rate(big_cfg, 1, budget_s=30.0, warmup=1)
        per_step = 24 / small + 8 / rate_b  # seconds per substep of every member
        agg = 32 / per_step
        line = {"metric": "substeps_per_s", "value": agg, "unit": unit, "impl": "reference", "n_gpus": args.gpus,
                "steps": n, "warmup": w, "ms_per_step": 1000.0 * 32 / agg, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": label, "members": 32},
                "cpu_baseline": {"value": agg, "unit": unit, "cores": threads, "kind": "port",
                                 "sample": f"{n} + {nb} substeps of a small and a large member (oracle, all host "
                                           f"threads), the members taken one after another"},
                "e2e": {"value": agg, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    rate_b, rate_c, rate_s, ms_b, ok = run_ensemble(args, local)
    ms = reduce_max(ms_b, dist, f"cuda:{local}")
    value = whole_job_rate(world, 3 * 32 * args.steps, ms)
    if rank == 0:
        line = {"metric": "substeps_per_s", "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
                "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if args.precision == "mixed" else "f64",
                "data": "synthetic",
                "config": {"workload": label, "members": 32, "precision": args.precision,
                           "form": "one ensemble context per member shape (24 and 8 members), each kernel of the "
                                   "substep covering all of its members in one launch",
                           "per_member_streams_substeps_per_s": rate_c,
                           "sequential_members_substeps_per_s": rate_s,
                           "l2": "inputs larger than L2 (no flush)"},
                "finite": ok}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def time_steps(s, dt, steps, stream, barrier, clocks=None):
    """`steps` time steps of context s between two CUDA events on its stream,
    with a barrier and a device synchronisation on both sides; returns the
    milliseconds, the per-kernel device times and the kernel launches."""
    import torch
    barrier()
    launches0 = s.launches
    s.reset_kernel_times()
    s.set_profiling(True)
    if clocks is not None:
        clocks.start()
        time.sleep(0.3)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        s.timestep(dt)
    e1.record(stream)
    e1.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop() if clocks is not None else None
    s.set_profiling(False)
    kt = {k: v for k, v in s.kernel_times().items() if v[1] > 0}
    if not math.isfinite(s.cfl):
        raise SystemExit("non-finite CFL: the run blew up")
    return ms, kt, s.launches - launches0, clk


def roofline(deck, s, kt, mixed, sub_ms, config):
    """The top kernel's roofline (its algorithmic bytes per launch over its
    average launch time, against the measured HBM copy bandwidth) and the
    whole substep's (B_alg over the substep time)."""
    per_kernel, b_sub, Ns, Nzx = alg_bytes(deck, s.nxd, s.nzd, kt.get("rhs", (0, 0))[1] > 0, mixed,
                                           kt.get("shift", (0, 0))[1] > 0)
    peak, peak_kind = peaks()
    top = max(kt, key=lambda k: kt[k][0])
    avg_ms = kt[top][0] / kt[top][1]
    achieved = per_kernel[top] / (avg_ms / 1000.0) / 1e9
    traffic = None
    tf = ROOT / "profiles" / f"traffic_{config}{'_mixed' if mixed else ''}.json"
    if tf.exists():
        traffic = json.loads(tf.read_text()).get(top)
    roof = {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_kind": peak_kind, "traffic": traffic, "alg_bytes_per_launch": per_kernel[top],
            "avg_launch_ms": avg_ms}
    sub = {"alg_bytes": b_sub, "ms_per_substep": sub_ms, "achieved_gbs": b_sub / (sub_ms / 1000.0) / 1e9,
           "frac": b_sub / (sub_ms / 1000.0) / 1e9 / peak}
    return roof, sub, {k: v[0] / v[1] for k, v in kt.items()}, {k: v[0] / sum(x[0] for x in kt.values())
                                                                for k, v in kt.items()}


def reference_main(args, cfg):
    """--impl reference: the oracle port of the reference's CPU path on all
    host threads, rank 0 only; each step is one substep of the workload from
    its seeded field (W warm-up substeps, then K timed)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    unit = "substeps/s"
    if not cfg.get("cpu_baseline", True):
        print(json.dumps({"impl": "reference", "unavailable": "one oracle substep of this workload needs more host "
                                                              "memory than the box is assumed to have"}), flush=True)
        return 0
    rate, threads, _, _ = oracle_substeps(cfg, args.warmup, args.steps)
    line = {"metric": "substeps_per_s", "value": rate, "unit": unit, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / rate, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": cfg["label"], "step": "one substep of the workload (a bounded sample; the "
                                                         "GPU arm's steps are whole RK3 time steps of 3 substeps)"},
            "cpu_baseline": {"value": rate, "unit": unit, "cores": threads, "kind": "port",
                             "sample": f"{args.steps} substeps of the workload from its seeded field after "
                                       f"{args.warmup} warm-up substeps (the oracle restatement of the reference "
                                       f"CPU path on {threads} threads; the Fortran+MPI+FFTW build is not "
                                       f"buildable in this image)"},
            "e2e": {"value": rate, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3", choices=sorted(CONFIGS) + ["c4"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="precision of the ensemble members (--config c4)")
    ap.add_argument("--sizes", default=None,
                    help="NX,NY,NZ: the workload's deck with other sizes (a smaller case of the same kernels, "
                         "for profiler captures); no CPU leg")
    args = ap.parse_args()
    if args.config == "c4":
        return ensemble_main(args)
    cfg = CONFIGS[args.config]
    cfg = dict(cfg, cpu_baseline=ORACLE_SUBSTEPS[args.config] > 0)
    if args.sizes:
        nx, ny, nz = (int(v) for v in args.sizes.split(","))
        cfg = dict(cfg, deck=dict(cfg["deck"], nx=nx, ny=ny, nz=nz), cpu_baseline=False,
                   label=cfg["label"] + f"; sizes replaced by nx={nx}, ny={ny}, nz={nz}")
        args.no_cpu_baseline = True
    if args.impl == "reference":
        return reference_main(args, cfg)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    metric, unit = "substeps_per_s", "substeps/s"

    import torch
    from homogenenousshearturbulence_b200 import hst
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = local
    torch.cuda.set_device(dev)
    deck = dict(cfg["deck"])
    dt = deck["deltat"]
    n_acc = ORACLE_SUBSTEPS[args.config] if (world == 1 and not args.no_cpu_baseline) else 0
    gpu_acc = {}

    def barrier_of(s):
        def barrier():
            torch.cuda.synchronize(dev)
            s.sync()
            if dist is not None:
                dist.barrier()
        return barrier

    # ---- the FP64 drop-in (the headline)
    s = hst.Solver(deck, device=dev)
    V0 = seeded_field(cfg, s.y)
    stream = torch.cuda.ExternalStream(s.stream, device=torch.device("cuda", dev))
    barrier = barrier_of(s)
    if n_acc:
        s.time = 0.0
        s.set_velocity(V0)
        s.timesteps(n_acc // 3, dt)
        gpu_acc["fp64"] = s.velocity()
    s.time = 0.0
    s.set_velocity(V0)
    for _ in range(args.warmup):
        s.timestep(dt)
    ms, kt, launches, clk = time_steps(s, dt, args.steps, stream, barrier, ClockSampler(dev))
    ms = reduce_max(ms, dist, f"cuda:{dev}")
    nsub = 3 * args.steps
    value = whole_job_rate(world, nsub, ms)

    # end to end through the public API with host buffers: every step
    # uploads the three velocity components from pinned memory, advances
    # one time step and downloads the three components (its result) into
    # other pinned buffers; the asynchronous I/O calls stage each upload in
    # device memory, so that the copy-in of one step runs beside the compute
    # of the previous one and beside the copy-out (the fixed-dt deck does
    # not read the CFL number back every step; it is read once at the end)
    e2e = None
    if not args.no_e2e:
        nbytes = s.shape[0] * s.shape[1] * s.shape[2] * 16
        pin_in = [torch.empty(nbytes, dtype=torch.uint8, pin_memory=True) for _ in range(3)]
        pin_out = [torch.empty(nbytes, dtype=torch.uint8, pin_memory=True) for _ in range(3)]
        for c in range(3):
            s.download_ptr(c, pin_in[c].data_ptr())
        ke = max(3, args.steps // 2)
        # one untimed round trip allocates the device snapshots
        for c in range(3):
            s.upload_async_ptr(c, pin_in[c].data_ptr())
        s.timesteps(1, dt)
        for c in range(3):
            s.download_async_ptr(c, pin_out[c].data_ptr())
        s.wait_io()
        barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(ke):
            for c in range(3):
                s.upload_async_ptr(c, pin_in[c].data_ptr())
            s.timesteps(1, dt)
            for c in range(3):
                s.download_async_ptr(c, pin_out[c].data_ptr())
        s.wait_io()
        f1.record(stream)
        f1.synchronize()
        mse = f0.elapsed_time(f1)
        if not math.isfinite(s.compute_cfl()):
            raise SystemExit("non-finite CFL after the end-to-end steps")
        mse = reduce_max(mse, dist, f"cuda:{dev}")
        e2e = {"value": whole_job_rate(world, 3 * ke, mse), "unit": unit, "h2d_bytes_per_step": 3 * nbytes,
               "d2h_bytes_per_step": 3 * nbytes, "steps": ke}
        del pin_in, pin_out
    roof, sub_roof, kms, kshare = roofline(deck, s, kt, False, ms / nsub, args.config)
    nxd, nzd = s.nxd, s.nzd
    s.close()

    # ---- the mixed-precision form on the same field
    mixed = None
    if not args.no_mixed:
        m = hst.Solver(dict(deck, precision="mixed"), device=dev)
        mstream = torch.cuda.ExternalStream(m.stream, device=torch.device("cuda", dev))
        if n_acc:
            m.time = 0.0
            m.set_velocity(V0)
            m.timesteps(n_acc // 3, dt)
            gpu_acc["mixed"] = m.velocity()
        m.time = 0.0
        m.set_velocity(V0)
        for _ in range(args.warmup):
            m.timestep(dt)
        mms, mkt, mlaunches, _ = time_steps(m, dt, args.steps, mstream, barrier_of(m))
        mms = reduce_max(mms, dist, f"cuda:{dev}")
        mroof, msub, mkms, _ = roofline(deck, m, mkt, True, mms / nsub, args.config)
        mixed = {"value": whole_job_rate(world, nsub, mms), "unit": unit, "ms_per_step": mms / args.steps,
                 "speedup_vs_fp64": ms / mms, "dtype": "f32+f64",
                 "form": "FP32 x-z transforms, products and product spectra; FP64 right-hand sides, shift, solves "
                         "and u, w",
                 "roofline": mroof, "substep_roofline": msub, "kernels_ms_per_launch": mkms,
                 "gpu_launches": mlaunches}
        m.close()

    if rank == 0:
        line = {
            "metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": cfg["label"], "precision": "fp64",
                       "step": "one RK3 time step = 3 substeps (hst_gpu_timestep)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single field, 1 GPU",
                       "l2": "inputs larger than L2 (no flush)", "nxd": nxd, "nzd": nzd},
            "roofline": roof, "substep_roofline": sub_roof,
            "kernels_ms_per_launch": kms, "kernel_share": kshare,
            "gpu_launches": launches,
            "clocks": clk,
        }
        if e2e:
            line["e2e"] = e2e
        if mixed:
            line["mixed"] = mixed
        if n_acc:
            # the oracle from the same seeded field: one warm-up substep, the
            # rest timed (the CPU baseline), its final velocity the reference
            # of both forms' accuracy after the same substeps
            rate, threads, Vo, _ = oracle_substeps(cfg, 1, n_acc - 1, V0)
            line["cpu_baseline"] = {"value": rate, "unit": unit, "cores": threads, "kind": "port",
                                    "sample": f"{n_acc - 1} substeps of the same workload from its seeded field "
                                              f"after 1 warm-up substep, oracle restatement of the reference CPU "
                                              f"path, {threads} threads"}

            def rel_l2(a, b):
                a, b = a[..., 2:-2], b[..., 2:-2]
                return float(np.linalg.norm(a - b) / np.linalg.norm(b))

            acc = {"substeps": n_acc, "against": "the oracle (FP64 CPU restatement of the reference path) from "
                                                 "the same seeded field, relative L2 over the interior rows"}
            for k, Vg in gpu_acc.items():
                acc[f"{k}_rel_l2_vs_oracle"] = rel_l2(Vg, Vo)
            line["accuracy"] = acc
            if mixed and "mixed" in gpu_acc:
                mixed["rel_l2_vs_oracle"] = acc["mixed_rel_l2_vs_oracle"]
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0

if __name__ == "__main__":
    sys.exit(main())
