"""Benchmark of the fused DG-SEM Maxwell LSRK45 path (libnwb) on B200.

Default workload (one GPU): periodic box [0,1]^3, 32x32x32 hexahedra, 8 GLL
points per direction (order 7, 16.8 M nodes x 6 fields = 100.7 M DOF), central
flux, CFL 0.5, Gaussian pulse Ez = exp(-|r-r0|^2/sigma^2), sigma = 0.1,
r0 ~ U[0.3,0.7]^3 from the seed.  A "step" is one LSRK45 time step (five fused
stage launches).  Other workloads: --workload c3 (PEC cavity 64x64x32, 6 points,
upwind), batch (256 uneven PEC cavities in one pool), serve (Poisson stream of
cavity solves, latency percentiles).

metric: GDOF-stage/s = 6 * npts * 5 * steps / seconds / 1e9.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|fp32]
                  [--workload c2|c3|batch|serve] [--accuracy-steps S]
  python bench.py --impl reference ...   # the reference's own CPU implementation

With --gpus N > 1 (under torchrun) every rank advances its own independent
cavity (replicas, weak scaling, no data-path collective); the timing is the
maximum over ranks and ``value`` is the sum of all ranks' DOF-stages over it.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GDOF-stage/s"
WORKLOAD = dict(workload="periodic_box_32x32x32_N8_central", nel=(32, 32, 32), N=8,
                periodic=True, c0=0.0, cfl=0.5, sigma=0.1)
BYTES_PER_DOF_STAGE = 32  # FP64 u and k, each read and written once


def workload_spec(name, nel_override, seed):
    """Single-mesh workloads c2 (the headline) and c3 (nekwave_b200.workloads)."""
    from nekwave_b200.workloads import single_mesh
    return single_mesh(name, nel_override, seed)


L2_BYTES = 126 * 1024 * 1024


def max_over_ranks(x: float, device: str = "cuda") -> float:
    """Largest value of x over all ranks (the job's time is its slowest rank's);
    x itself without a process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(dof_stages_per_rank: float, seconds_max: float, world: int) -> float:
    """Whole-job GDOF-stage/s: every rank's DOF-stages over the slowest rank's time."""
    return dof_stages_per_rank * world / seconds_max / 1e9


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=500)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["nwb", "reference"], default="nwb")
    p.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--e2e-steps", type=int, default=10)
    p.add_argument("--nel", type=int, default=32,
                   help="elements per axis; values other than 32 are for profiling only")
    p.add_argument("--variant", type=int, default=-1,
                   help="stage-kernel launch shape; -1 = autotune on the workload")
    p.add_argument("--workload", choices=["c2", "c3", "batch", "serve"], default="c2",
                   help="c2: periodic 32^3 N=8 (default, the headline); batch: 256 uneven PEC "
                        "cavities in one pool; serve: Poisson request stream")
    p.add_argument("--rates", type=str, default="0.25,0.5,1,2,4",
                   help="serve: arrival rates as multiples of the measured serial service rate")
    p.add_argument("--requests", type=int, default=100, help="serve: requests per rate")
    p.add_argument("--policies", type=str, default="fifo,sjf", help="serve: admission policies")
    p.add_argument("--serial-replay", action="store_true",
                   help="serve: replay the stream in real time on the serial path at every rate "
                        "(default: its schedule from service times measured once)")
    p.add_argument("--t-scale", type=float, default=1.0,
                   help="serve: final times T ~ U[0.5,2] scaled by this factor (fewer steps per "
                        "request; same sizes and orders)")
    p.add_argument("--serial-rate-per-s", type=float, default=0.0,
                   help="serve: the serial service rate (solves/s) to scale the arrivals by, "
                        "instead of measuring it (lets a sweep be split over runs)")
    p.add_argument("--accuracy-steps", type=int, default=0,
                   help="c2: also run FP64 and FP32-bulk this many steps from the same initial "
                        "state and report the relative L2 error and energy drift")
    p.add_argument("--profile", action="store_true",
                   help="only warm-up + timed steps (small case for ncu captures)")
    return p.parse_args()


def initial_state(x, y, z, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    r0 = rng.uniform(0.3, 0.7, 3)
    n = x.size
    u = np.zeros(6 * n)
    s2 = WORKLOAD["sigma"] ** 2
    u[2 * n:3 * n] = np.exp(-((x - r0[0]) ** 2 + (y - r0[1]) ** 2 + (z - r0[2]) ** 2) / s2)
    return u


# ---- clocks ------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except FileNotFoundError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            f = [c.strip() for c in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5], f[6], f[7], f[8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[2:]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(r[0] for r in rows),
                "sm_max_mhz": max(r[1] for r in rows), "samples": len(rows),
                "reasons": sorted(reasons)}


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(N):
    """DRAM bytes per stage launch from the committed ncu summary of the stage kernel
    with N points per direction, if any (stage_kernel_traffic.json covers N=8,
    stage_kernel_traffic_n<N>.json the others)."""
    for name in ("stage_kernel_traffic.json", f"stage_kernel_traffic_n{N}.json"):
        try:
            with open(os.path.join(ROOT, "profiles", name)) as f:
                d = json.load(f)
        except (OSError, ValueError):
            continue
        if int(d.get("N", 8)) == N:
            return d
    return None


def pool_traffic(seed):
    """DRAM bytes of one pool stage (all per-N kernels) on the 256-cavity workload of
    seed 0, from the committed ncu summary (pool_step_traffic.json), or None."""
    if seed != 0:
        return None
    try:
        with open(os.path.join(ROOT, "profiles", "pool_step_traffic.json")) as f:
            return float(json.load(f)["dram_bytes_per_stage"])
    except (OSError, ValueError, KeyError):
        return None


# ---- CPU baseline: the reference's own implementation on the host cores ---------------
def _sample_mesh(spec, O):
    """An 8x8x8-element sub-box of the workload with the same points per direction,
    boundary kind and flux, built by the reference's own Mesh when available."""
    N = spec["N"]
    nel = (8, 8, 8)
    lo = np.array(spec["lo"])
    h = (np.array(spec["hi"]) - lo) / np.array(spec["nel"])
    hi = lo + h * np.array(nel)
    per = spec["periodic"]
    if O.ref_available():
        m = O.ref_box_mesh(N, nel, tuple(lo), tuple(hi), per)
        return m, m.dxmin_ref, O.ref_step, O.ref().nwref_threads(), "reference"
    m = O.box_mesh(N, nel, tuple(lo), tuple(hi), per)
    return m, O.dxmin(m), O.step, O.threads(), "port"


def cpu_reference_rate(seconds_target=12.0, spec=None, one_core=0.0):
    """Times the reference's RHS + LSRK45 (its kernel bodies compiled for the host,
    oracle/_ref) -- or, if that build is absent, the oracle port -- on a bounded sample
    of the workload: whole LSRK45 steps on an 8x8x8-element sub-box with the same
    points per direction, boundaries and flux."""
    from oracle import oracle as O
    spec = spec or workload_spec("c2", 32, 0)
    m, dx, stepper, cores, kind = _sample_mesh(spec, O)
    u = np.random.Generator(np.random.PCG64(1)).standard_normal(6 * m.npts)
    dt = WORKLOAD["cfl"] * dx
    t0 = time.perf_counter()
    u, k = stepper(m, spec["c0"], dt, 1, u)
    one = time.perf_counter() - t0
    nsteps = max(1, int(seconds_target / max(one, 1e-3)))
    t0 = time.perf_counter()
    stepper(m, spec["c0"], dt, nsteps, u, k)
    sec = time.perf_counter() - t0
    dof_stage = 6 * m.npts * 5 * nsteps
    out = dict(value=dof_stage / sec / 1e9, unit=METRIC, cores=int(cores), kind=kind,
               sample=f"{nsteps} LSRK45 steps on an 8x8x8-element sub-box of the workload, "
                      f"N={spec['N']} ({m.npts} nodes), {sec:.1f} s on {cores} host threads",
               seconds=sec, steps=nsteps, npts=m.npts, cpu_model=cpu_model())
    if one_core and kind == "reference" and cores > 1:
        # the same sample on one host thread, a bounded number of steps
        old = O.ref().nwref_set_threads(1)
        try:
            n1 = max(1, int(one_core / max(one * cores, 1e-3)))
            t0 = time.perf_counter()
            stepper(m, spec["c0"], dt, n1, u, k)
            s1 = time.perf_counter() - t0
        finally:
            O.ref().nwref_set_threads(old)
        out["one_core"] = dict(value=6 * m.npts * 5 * n1 / s1 / 1e9, unit=METRIC, cores=1,
                               sample=f"{n1} LSRK45 steps of the same sub-box, {s1:.1f} s on 1 "
                                      f"host thread")
    return out


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), or None."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def run_reference(args, rank, world):
    """--impl reference: the reference's own CPU implementation (oracle/_ref), each
    step one LSRK45 step of an 8x8x8-element sub-box of the workload."""
    if rank != 0:
        return None
    from oracle import oracle as O
    spec = workload_spec(args.workload if args.workload in ("c2", "c3") else "c2", args.nel, args.seed)
    m, dx, stepper, cores, kind = _sample_mesh(spec, O)
    u = np.random.Generator(np.random.PCG64(1)).standard_normal(6 * m.npts)
    k = np.zeros_like(u)
    dt = WORKLOAD["cfl"] * dx
    for _ in range(args.warmup):
        u, k = stepper(m, spec["c0"], dt, 1, u, k)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        u, k = stepper(m, spec["c0"], dt, 1, u, k)
        times.append(time.perf_counter() - t0)
    sec = sum(times)
    value = 6 * m.npts * 5 * args.steps / sec / 1e9
    sample = (f"each step: one LSRK45 step on an 8x8x8-element sub-box of the workload, "
              f"N={spec['N']} ({m.npts} nodes)")
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sec / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(workload=spec["workload"], N=spec["N"], nel=list(spec["nel"]),
                           flux=spec["flux"], cfl=WORKLOAD["cfl"], sample_nel=[8, 8, 8]),
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": int(cores), "kind": kind,
                             "sample": sample, "cpu_model": cpu_model()},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def run_batch(args, rank, world):
    """256 PEC cavities (uneven sizes, 4..9 points) advanced together in one pool:
    one persistent launch per LSRK stage, one CUDA graph per step."""
    import torch
    from nekwave_b200 import DgSolver
    from nekwave_b200.pool import CavityPool
    from nekwave_b200.workloads import batch_instances
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    inst = batch_instances(256, seed=args.seed + rank, steps=args.steps)
    budget = int(sum(3 * 6 * c.npts * 8 + c.nel[0] * c.nel[1] * c.nel[2] * 400 for c in inst) * 1.2
                 + (1 << 30))
    prec = args.precision
    pool = CavityPool(budget, max_slots=len(inst), precision=prec)
    slots = [pool.add_box(c.N, c.nel, c.lo, c.hi, c.c0, c.dt, c.nsteps, energy_every=50)
             for c in inst]
    for s, c in zip(slots, inst):
        pool.init_pulse(s, c.pulses)
    mode, mode_ms = pool.autotune(reps=5)
    pool.step(args.warmup)
    pool.sync()
    for s, c in zip(slots, inst):          # back to t = 0 for the timed run
        pool.init_pulse(s, c.pulses)
    launches0 = pool.info()["launches"]
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        torch.cuda.synchronize()
        ms = pool.time_steps(args.steps)
        torch.cuda.synchronize()
    launches = pool.info()["launches"] - launches0
    total = sum(c.dof_stages for c in inst)
    value = total / (ms / 1e3) / 1e9
    finals = {s: pool.results(s, energy=False, probes=False)["state"] for s in slots[:32]}
    pool.close()
    # per-instance error of this precision against an FP64 pool (first 32 instances)
    errs = []
    if prec != "fp64":
        ref = CavityPool(budget, max_slots=32, precision="fp64")
        rs = [ref.add_box(c.N, c.nel, c.lo, c.hi, c.c0, c.dt, c.nsteps, energy_every=50)
              for c in inst[:32]]
        for s, c in zip(rs, inst[:32]):
            ref.init_pulse(s, c.pulses)
        ref.step(args.steps)
        for s_ref, s in zip(rs, slots[:32]):
            a = ref.results(s_ref, energy=False, probes=False)["state"]
            errs.append(float(np.linalg.norm(finals[s] - a) / np.linalg.norm(a)))
        ref.close()
    # serial plain FP64 single-mesh path on the same instances (bounded sample)
    ser_dof, ser_ms = 0, 0.0
    for c in inst[:48]:
        so = DgSolver("fp64")
        so.initializeBox(c.N, c.nel, c.lo, c.hi, c.c0)
        so.initPulse(c.pulses)
        so.steps(c.dt, 3)
        ser_ms += so.timeSteps(c.dt, c.nsteps, graph=True)
        ser_dof += c.dof_stages
        so.finalize()
    serial = ser_dof / (ser_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    achieved = BYTES_PER_DOF_STAGE * total / 5 / args.steps / (ms / 1e3 / args.steps / 5) / 1e9
    return {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == "fp64" else "f32-bulk/f64-lsrk", "data": "synthetic (seeded)",
            "config": dict(workload="batch_256_pec_cavities", instances=len(inst),
                           launch_mode=("one launch per N" if mode else "one persistent launch"),
                           autotune_stage_ms=mode_ms,
                           nodes=int(sum(c.npts for c in inst)), points_per_dir="4..9",
                           elements_per_dir="2..12", steps_each=args.steps, precision=prec,
                           l2="inputs larger than L2 (3 x %.2f GB)" % (
                               sum(c.npts for c in inst) * 48 / 1e9)),
            "gpu_launches": int(launches), "clocks": clk.summary(),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": pool_traffic(seed=args.seed + rank),
                         "peak_source": peak_kind,
                         "kernel": "one stage: the per-N stage kernels of every N present",
                         "per_unit": "32 B per DOF-stage x 6 x nodes (all cavities) per stage"},
            "serial_fp64_single_mesh": {"value": serial, "unit": METRIC,
                                        "sample": "first 48 instances solved one at a time with "
                                                  "the single-mesh FP64 solver (CUDA graph per step)",
                                        "speedup_batched": value / serial},
            "error_vs_fp64": ({"rel_l2_max": max(errs), "rel_l2_median": float(np.median(errs)),
                               "instances": len(errs)} if errs else None)}


def run_serve(args, rank, world):
    """Poisson stream of cavity solves served with continuous batching; p50/p99
    latency and solves/s per arrival rate, next to the serial FP64 path.

    The serial path takes one request at a time in arrival order, so its schedule
    follows from each request's service time: finish_i = max(arrival_i,
    finish_{i-1}) + service_i.  The service times are measured once, the requests
    run back to back on the single-mesh solver (serving.serial_service_times), and
    the serial latencies at every rate come from that schedule; --serial-replay
    instead replays the stream in real time at each rate."""
    import torch
    from nekwave_b200.serving import (Server, fifo_finish_times, latency_stats, latency_summary,
                                      serial_service_times, serve_serial)
    from nekwave_b200.workloads import serving_requests
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n = args.requests
    base = serving_requests(n, 1.0, seed=args.seed + 100, t_scale=args.t_scale)  # arrivals at 1/s
    work = sum(c.dof_stages for c in base)
    budget = int(float(os.environ.get("NWB_SERVE_BUDGET_GB", "100")) * (1 << 30))
    if args.serial_rate_per_s > 0:
        svc = None
        mu = args.serial_rate_per_s
    else:
        solve_warm = serving_requests(2, 1.0, seed=args.seed + 1000, t_scale=0.05)
        serial_service_times(solve_warm)                     # first-use set-up off the clock
        svc = serial_service_times(base)
        mu = n / float(svc.sum())                            # serial solves/s on this request set
    rates = [float(x) for x in args.rates.split(",")]
    rows = []
    for mult in rates:
        reqs = [dataclasses.replace(r, arrival=r.arrival / (mult * mu)) for r in base]
        for policy in [x for x in args.policies.split(",") if x]:
            srv = Server(budget, max_slots=512, precision=args.precision, policy=policy)
            res, wall = srv.run(reqs)
            srv.close()
            st = latency_stats(res)
            rows.append(dict(policy=policy, rate_multiple=mult, rate_per_s=mult * mu,
                             solves_per_s=n / wall, p50_s=st["p50"], p99_s=st["p99"],
                             mean_s=st["mean"], max_s=st["max"],
                             gdof_stage_per_s=work / wall / 1e9))
    serial = []
    for mult in rates:
        arr = np.array([r.arrival / (mult * mu) for r in base])
        if args.serial_replay or svc is None:
            serial_reqs = [dataclasses.replace(r, arrival=a) for r, a in zip(base, arr)]
            sres, swall = serve_serial(serial_reqs, precision="fp64")
            sst = latency_stats(sres)
            how = "replayed in real time"
        else:
            fin = fifo_finish_times(arr, svc)
            sst = latency_summary(fin - arr)
            swall = float(fin.max())
            how = "schedule from the measured service times"
        serial.append(dict(rate_multiple=mult, rate_per_s=mult * mu, solves_per_s=n / swall,
                           p50_s=sst["p50"], p99_s=sst["p99"], mean_s=sst["mean"],
                           max_s=sst["max"], gdof_stage_per_s=work / swall / 1e9, how=how))
    best = max(rows, key=lambda r: r["solves_per_s"]) if rows else {"solves_per_s": None}
    return {"metric": "solves/s", "value": best["solves_per_s"], "unit": "solves/s", "n_gpus": world,
            "steps": n, "warmup": 0, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32-bulk/f64-lsrk",
            "data": "synthetic Poisson stream (seeded)",
            "config": dict(workload="serving_poisson_pec_cavities", requests_per_rate=n,
                           final_time_scale=args.t_scale,
                           serial_service_rate_per_s=mu,
                           serial_gdof_stage_per_s=(mu * work / n / 1e9),
                           mean_request_gdof_stage=work / n / 1e9, max_elements_per_dir=48,
                           points_per_dir="4..9", budget_gb=budget / (1 << 30),
                           serial_service_s=(dict(p50=float(np.median(svc)), mean=float(svc.mean()),
                                                  max=float(svc.max())) if svc is not None else None)),
            "serving": rows,
            "serial_fp64": serial,
            "serial_pattern": "one request at a time with the single-mesh FP64 solver, a step at a "
                              "time, the 8 probes read after every step and the energy every 10 "
                              "steps (the reference's Case::simulate loop, diagnostics on the device)"}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    if args.workload in ("batch", "serve"):
        fn = run_batch if args.workload == "batch" else run_serve
        line = fn(args, rank, world)
        if rank == 0:
            print(json.dumps(line), flush=True)
        return

    import torch
    import torch.distributed as dist
    from nekwave_b200 import DgSolver

    torch.cuda.set_device(local)
    dist_on = world > 1
    if dist_on:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist_on:
            dist.barrier()
        torch.cuda.synchronize()

    spec = workload_spec(args.workload, args.nel, args.seed + rank)
    N, nel = spec["N"], spec["nel"]
    npts = nel[0] * nel[1] * nel[2] * N ** 3
    from nekwave_b200.workloads import box_dxmin
    dt = WORKLOAD["cfl"] * box_dxmin(N, nel, spec["lo"], spec["hi"])
    pulses = spec["pulses"]
    solver = DgSolver(args.precision)
    solver.initializeBox(N, nel, spec["lo"], spec["hi"], spec["c0"], periodic=spec["periodic"])
    solver.initPulse(pulses)
    u0 = solver.downloadState()
    tune_ms = None
    if args.variant >= 0:
        solver.setVariant(args.variant)
    else:
        _, tune_ms = solver.autotune(reps=10)
    info = solver.info()

    # warm-up (graphs captured here)
    solver.steps(dt, args.warmup)
    barrier()
    if args.profile:
        solver.steps(dt, args.steps)
        barrier()
        print(json.dumps({"profile": True, "nel": nel, "npts": npts, "steps": args.steps,
                          "energy": solver.energy()}))
        solver.finalize()
        return

    # ---- timed region: K steps, inputs resident in HBM (u_in, u_out, k each > L2) -------
    launches0 = solver.launchCount()
    with ClockSampler(local) as clk:
        barrier()
        ms = solver.timeSteps(dt, args.steps, graph=True)
        barrier()
    launches = solver.launchCount() - launches0
    clocks = clk.summary()
    ms_max = max_over_ranks(ms)
    value = job_rate(6 * npts * 5 * args.steps, ms_max / 1e3, world)

    # ---- roofline of the fused stage kernel (CUDA events on the solver's stream) ----------
    stage_ms = solver.timeStageKernel(dt, 50)
    alg_bytes = BYTES_PER_DOF_STAGE * 6 * npts
    achieved = alg_bytes / (stage_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    tr = profiled_traffic(N)
    traffic = None
    # the committed capture is of the default shape (variant 0) in one precision
    if (tr and tr.get("npts") and tr.get("precision", "fp64") == args.precision
            and solver.info()["variant"] == 0):
        traffic = tr["dram_bytes_per_launch"] * npts / tr["npts"]

    # ---- end to end through the public API, host buffers, copies inside the timed region --
    import ctypes
    host = torch.empty(6 * npts, dtype=torch.float64).pin_memory()
    host.copy_(torch.from_numpy(u0))
    hnp = host.numpy()
    e2e_steps = args.e2e_steps
    # (1) the reference's blocking calls: upload, step, download, one after another
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        solver.uploadState(hnp)            # H2D of the step's input state (pinned)
        solver.step(dt, 0.0)               # one LSRK45 step (blocking, as the reference)
        solver.downloadState(hnp)          # D2H of the step's result state
    barrier()
    e2e_block = job_rate(6 * npts * 5 * e2e_steps, max_over_ranks(time.perf_counter() - t0), world)
    # (2) the same copies pipelined: each step's input state is uploaded
    # asynchronously (host -> staging on an upload stream while the previous step
    # runs, then staging -> state in stream order) and its result leaves through the
    # asynchronous snapshot (device copy in stream order, then device -> host on a
    # side stream), so the host link carries step i+1's input and step i's result at
    # the same time while the GPU steps; the last snapshot is waited for inside the
    # timed region.  Every step still moves its whole input in and its whole result out.
    host_out = torch.empty(6 * npts, dtype=torch.float64).pin_memory()
    hout = host_out.numpy()
    solver.snapshotBegin(hout)             # set-up of the snapshot and staging buffers, untimed
    solver.snapshotWait()
    solver.uploadBegin(hnp)
    solver.uploadWait()
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        solver.uploadBegin(hnp)            # H2D of the step's input state (pinned)
        solver.steps(dt, 1, sync=False)    # one LSRK45 step, queued behind the upload
        solver.snapshotBegin(hout)         # D2H of the step's result state
    solver.snapshotWait()
    solver.uploadWait()
    barrier()
    e2e_value = job_rate(6 * npts * 5 * e2e_steps, max_over_ranks(time.perf_counter() - t0), world)
    del ctypes, host_out

    accuracy = None
    if args.accuracy_steps > 0:
        out = {}
        for prec in ("fp64", "fp32"):
            a = DgSolver(prec)
            a.initializeBox(N, nel, spec["lo"], spec["hi"], spec["c0"], periodic=spec["periodic"])
            a.initPulse(pulses)
            e0 = a.energy()
            a.steps(dt, args.accuracy_steps)
            out[prec] = (a.downloadState(), e0, a.energy())
            a.finalize()
        u64, u32 = out["fp64"][0], out["fp32"][0]
        accuracy = {"steps": args.accuracy_steps,
                    "fp32_rel_l2_vs_fp64": float(np.linalg.norm(u32 - u64) / np.linalg.norm(u64)),
                    "energy_drift_fp64": (out["fp64"][2] - out["fp64"][1]) / out["fp64"][1],
                    "energy_drift_fp32": (out["fp32"][2] - out["fp32"][1]) / out["fp32"][1]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_rate(spec=spec, one_core=6.0)

    if dist_on:
        dist.barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32-bulk/f64-lsrk",
            "data": "synthetic (seeded Gaussian pulse)",
            "config": dict(workload=spec["workload"], N=N, order=N - 1,
                           nel=list(nel), npts=npts, dof=6 * npts,
                           flux=spec["flux"], cfl=WORKLOAD["cfl"], dt=dt,
                           precision=args.precision, parallelism=f"replicas x{world}",
                           l2="inputs larger than L2 (u_in, u_out, k: 3 x %.0f MB)" % (npts * 48 / 1e6),
                           kernel=dict(variant=info["variant"], ks=info["ks"], epb=info["epb"],
                                       k_in_smem=info["ksmem"], minb=info["minb"],
                                       threads=info["threads_per_block"],
                                       smem=info["smem_bytes"], geometry=info["geometry"],
                                       autotune_ms=tune_ms)),
            "gpu_launches": int(launches),
            "clocks": clocks,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": peak_kind, "kernel": "stage_kernel",
                         "stage_ms": stage_ms, "alg_bytes_per_launch": alg_bytes},
            "e2e": {"value": e2e_value, "unit": METRIC,
                    "h2d_bytes_per_step": 6 * npts * 8, "d2h_bytes_per_step": 6 * npts * 8,
                    "steps": e2e_steps,
                    "pattern": "uploadBegin (asynchronous H2D of the step's input from pinned "
                               "memory) + step + snapshotBegin (asynchronous D2H of its result) per "
                               "step, pipelined so that step i+1's upload and step i's download "
                               "share the host link while the GPU steps; the last snapshot and "
                               "upload waited for inside the timed region",
                    "blocking": {"value": e2e_block, "pattern": "uploadState (pinned) + step + "
                                 "downloadState per step, the reference's blocking calls"}},
        }
        if accuracy is not None:
            line["accuracy"] = accuracy
        if cpu is not None:
            line["cpu_baseline"] = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample",
                                                          "cpu_model", "one_core") if k in cpu}
        print(json.dumps(line), flush=True)
    solver.finalize()
    if dist_on:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
