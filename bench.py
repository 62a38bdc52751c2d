#!/usr/bin/env python3
"""Benchmark of the uniform-grid PF-FLIP step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one Simulator.step over the whole particle set): the
128^3 dam break with 27 particles per cell (56,623,104 particles), liquid for
x < 0.4 and y < 0.6, 1000:1 density, fixed dt = 0.5 dx / sqrt(2 g 0.6),
MG-PCG to 1e-4 (the reference's production tolerance), plain FP32.  Seeding is
the reference's jittered lattice from seed 42 (synthetic, no dataset).

Printed (rank 0, one JSON line): steps/s of the whole job (``value``), the same
metric end to end through the public API with the particle state uploaded from
and read back to pinned host memory every step (``e2e``), the roofline of the
dominant kernel from CUDA events in the timed region, SM clocks sampled during
the timed region, this library's kernel launches in the timed region, the CPU
oracle timed on a bounded sample (``cpu_baseline``), the standalone 128^3 MG-PCG
solve to 1e-6 in FP32 and with the 16-bit hierarchy (``solve``), and the
mixed-precision step (``mixed``).

Multi-GPU: the step does not shard here (one GPU per simulation), so N ranks run
N independent replicas (weak scaling, no data-path collective); the timing is
the max over ranks.

``--impl reference`` times the reference algorithm's CPU restatement (the
oracle; NVIDIA Warp, the reference's runtime, is not installed) on the host
cores with all threads, on the same workload and metric.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "implementation-of-adaptive-phase-field-flip_b200"))
sys.path.insert(0, REPO)

METRIC = "steps/s, dam_break 128^3 27ppc (56.6M particles) 1000:1, full PF-FLIP step"
UNIT = "steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--res", type=int, default=128)
    ap.add_argument("--ppc", type=int, default=27)
    ap.add_argument("--tol", type=float, default=1e-4)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp16", "bf16"])
    ap.add_argument("--stencil", default="flux", choices=["flux", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-solve", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-solve-oracle", action="store_true",
                    help="skip the FP64 CG oracle (solved to 1e-12) that the solve leg's errors are measured against")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the step-accuracy leg (phi, pressure, divergence of the FP32/FP16/BF16 step vs FP64)")
    ap.add_argument("--solve-only", action="store_true", help="only the standalone solve leg (prints its JSON)")
    ap.add_argument("--solve-variants", default="fp32_flux,fp16_flux,bf16_flux,fp32_reference",
                    help="comma list of precision_stencil variants for the solve leg")
    ap.add_argument("--solve-repeats", type=int, default=5)
    ap.add_argument("--no-graphs", action="store_true", help="solve leg without CUDA graphs")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the differentiable-asteroid gradient leg")
    ap.add_argument("--adjoint-only", action="store_true", help="only the gradient leg (prints its JSON)")
    ap.add_argument("--adjoint-res", type=int, default=64)
    ap.add_argument("--adjoint-steps", type=int, default=20)
    ap.add_argument("--no-adjoint-fd", action="store_true",
                    help="skip the check of the gradient against FP64 central differences of the CPU oracle")
    ap.add_argument("--no-rt", action="store_true",
                    help="skip the Rayleigh-Taylor legs (256^3 forward, FP32 and 16-bit hierarchy; 128^3 a_k gradient)")
    ap.add_argument("--rt-grad-res", type=int, default=128)
    ap.add_argument("--rt-grad-steps", type=int, default=50)
    ap.add_argument("--no-rt-fd", action="store_true", help="skip the 32^3 FP64 finite-difference check of the a_k gradient")
    ap.add_argument("--rt-only", action="store_true", help="only the Rayleigh-Taylor leg (prints its JSON)")
    ap.add_argument("--rt-res", type=int, default=256)
    ap.add_argument("--adjoint-fd-res", type=int, default=None,
                    help="grid of the finite-difference check (default: --adjoint-res)")
    return ap.parse_args()


def workload_cfg(args, precision=None):
    from pfflip import Config

    r = args.res
    return Config(res=(r, r, r), dx=1.0 / r, ppc=args.ppc, seed=42, droplets=False, pcg_tol=args.tol,
                  precision=precision or args.precision, stencil=args.stencil)


def fixed_dt(dx):
    return 0.5 * dx / math.sqrt(2 * 9.81 * 0.6)


def seed_particles(cfg):
    from pfflip import scenes

    return scenes.dam_break(cfg)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        exe = shutil.which("nvidia-smi")
        if exe is None:
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.fh = open(self.path, "w")
        self.proc = subprocess.Popen([exe, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                      "-i", str(self.gpu), "-lms", "100"], stdout=self.fh,
                                     stderr=subprocess.DEVNULL)

    def stop(self):
        if self.proc is None:
            return {"samples": 0, "note": "nvidia-smi unavailable"}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        rows = []
        for ln in open(self.path):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), float(parts[3]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"samples": 0}
        sm = np.array([r[0] for r in rows])
        mx = max(r[1] for r in rows)
        load = sm[sm > 0.5 * mx] if (sm > 0.5 * mx).any() else sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[3]) if v.lower().startswith("active")})
        return {"sm_mhz": float(np.median(load)), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows),
                "power_w_max": max(r[2] for r in rows)}


# ---------------------------------------------------------------- algorithmic bytes
def algorithmic_bytes(stage, n_particles, n_cells, iters):
    """Bytes each stage must move, counting every array once per launch (the
    per-unit figures of the path's byte model; the float4 streams actually
    move 32 B per particle and direction)."""
    if stage == "p2g":  # read x,y,z,u,v,w + phase (25 B), write 8 accumulator grids (32 B/cell)
        return 25 * n_particles + 32 * n_cells
    if stage == "g2p_advect":  # read pos, vel, phase (25 B), write pos, vel (24 B); gathers L2-resident
        return 49 * n_particles
    if stage == "sort":  # key write+read x2, 25 B gather, 25 B scatter, 4 B permutation
        return 70 * n_particles
    if stage == "solve":  # ~ (V-cycle 205*8/7 + CG 68) B per cell and iteration
        return (205 * 8 / 7 + 68) * n_cells * max(iters, 1)
    return None


def load_traffic():
    p = os.path.join(REPO, "profiles", "traffic_per_unit.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except Exception:
            return {}
    return {}


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------- CPU oracle leg
def cpu_oracle_steps(cfg, pos, vel, pt, nsteps, threads):
    from oracle import oracle as O

    O.set_threads(threads)
    o = O.OracleSim(cfg, nthreads=threads, stencil=cfg.stencil)
    o.set_particles(pos, vel, pt)
    dt = fixed_dt(cfg.dx)
    times = []
    for _ in range(nsteps):
        t0 = time.perf_counter()
        o.step(dt)
        times.append(time.perf_counter() - t0)
    return times


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cfg = workload_cfg(args)
    pos, vel, pt = seed_particles(cfg)
    threads = os.cpu_count() or 1
    steps = max(1, min(args.steps, 2))
    warm = min(args.warmup, 1)
    probe = warp_probe()
    times = cpu_oracle_steps(cfg, pos, vel, pt, warm + steps, threads)[warm:]
    v = len(times) / sum(times)
    sample = (f"{len(times)} full oracle steps (after {warm} warm-up) of the {args.res}^3/{args.ppc}ppc dam break, "
              f"{len(pos):,} particles; reference runtime NVIDIA Warp unavailable on this box ({probe}), so the "
              f"CPU restatement of the reference kernels (oracle/pf_oracle.hpp) runs in its place")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": len(times), "warmup": warm, "ms_per_step": 1000.0 / v, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic", "config": {"workload": f"dam_break {args.res}^3 {args.ppc}ppc"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "warp_probe": probe}
    print(json.dumps(line), flush=True)
    return 0


def warp_probe():
    """Whether the reference's runtime (NVIDIA Warp, warp-lang) imports here:
    the exception's one-line text, or its version.  The reference package
    itself is not on this machine either way, so the oracle port stands in."""
    try:
        import warp  # noqa: F401
    except Exception as e:  # ModuleNotFoundError on these boxes
        return f"import warp: {type(e).__name__}: {e}"
    return f"import warp: ok, version {getattr(warp, '__version__', '?')}"


# ---------------------------------------------------------------- ranks
class Ranks:
    """Process-group plumbing of a run over N ranks (one process per GPU,
    launched by torch.distributed.run).  The step does not shard, so the ranks
    exchange no data: they meet at barriers around the timed region and reduce
    one number, the elapsed time (max over ranks).  Every rank takes the same
    collective calls in the same order.  ``backend`` is "nccl" on GPUs; the
    CPU tests drive the same code with "gloo"."""

    def __init__(self, backend, device):
        import torch

        self.torch = torch
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.device = device
        self.dist = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            kw = {"device_id": device} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300), **kw)
            self.dist = dist

    @property
    def root(self):
        return self.rank == 0

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()
        if self.device.type == "cuda":
            self.torch.cuda.synchronize(self.device)

    def max(self, x):
        """max of x over the ranks (x itself on one rank)"""
        if self.dist is None:
            return float(x)
        t = self.torch.tensor([float(x)], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def job_rate(world, ms_per_step_max):
    """whole-job steps/s of N replicas whose slowest rank took ms_per_step_max"""
    return world * 1000.0 / ms_per_step_max


# ---------------------------------------------------------------- GPU legs
def run_ours(args):
    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ranks = Ranks("nccl", torch.device("cuda", local))
    world, rank = ranks.world, ranks.rank
    barrier, max_over_ranks = ranks.barrier, ranks.max

    from pfflip import Simulator
    from pfflip import _native as N

    cfg = workload_cfg(args)
    dt = fixed_dt(cfg.dx)
    t_seed = time.perf_counter()
    pos, vel, pt = seed_particles(cfg)
    t_seed = time.perf_counter() - t_seed
    n = len(pos)
    ncell = cfg.res[0] * cfg.res[1] * cfg.res[2]

    sim = Simulator(cfg)
    sim.set_particles(pos, vel, pt)
    for _ in range(args.warmup):
        sim.step(dt)
    sim.enable_stage_timing(True)
    sim.stage_times(reset=True)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    l0 = N.launch_count()
    e0.record(stream)
    recs = [sim.step(dt) for _ in range(args.steps)]
    e1.record(stream)
    barrier()
    launches = N.launch_count() - l0
    clk = clocks.stop()
    ms_local = e0.elapsed_time(e1) / args.steps
    ms = max_over_ranks(ms_local)
    stages = sim.stage_times(reset=True)
    sim.enable_stage_timing(False)
    iters = float(np.mean([r["pcg_iter"] for r in recs]))
    value = job_rate(world, ms)

    # roofline of the dominant single-kernel stage
    peak, peak_kind = peaks()
    traffic_db = load_traffic()
    per_stage = {k: {"launches": c, "ms_per_launch": t / c, "share": t / (ms_local * args.steps)}
                 for k, (c, t) in stages.items()}
    single = [k for k in ("p2g", "g2p_advect") if k in per_stage]
    dom = max(single, key=lambda k: per_stage[k]["ms_per_launch"]) if single else None
    roof = None
    if dom:
        ab = algorithmic_bytes(dom, n, ncell, iters)
        dur = per_stage[dom]["ms_per_launch"] * 1e-3
        ach = ab / dur / 1e9
        tr = traffic_db.get(dom, {})
        traffic = None
        if "bytes_per_particle" in tr:
            traffic = tr["bytes_per_particle"] * n + tr.get("bytes_per_cell", 0.0) * ncell
        roof = {"kernel": {"p2g": "k_p2g", "g2p_advect": "k_g2p_advect_packed"}[dom], "bound": "hbm", "achieved": ach,
                "peak": peak, "unit": "GB/s", "frac": ach / peak, "peak_kind": peak_kind,
                "algorithmic_bytes_per_launch": ab, "traffic": traffic}
    for k, v in per_stage.items():
        ab = algorithmic_bytes(k, n, ncell, iters)
        if ab is not None:
            v["achieved_gbs"] = ab / (v["ms_per_launch"] * 1e-3) / 1e9
    sweep = sweep_roofline(sim, ncell, peak, peak_kind)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"dam_break {args.res}^3 {args.ppc}ppc", "res": args.res, "ppc": args.ppc,
                   "particles": n, "dt": dt, "pcg_tol": args.tol, "precision": args.precision,
                   "stencil": args.stencil, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (particle streams 2x1.8 GB)", "pcg_iter_mean": iters},
        "clocks": clk, "gpu_launches": int(launches), "roofline": roof, "roofline_solver_sweep": sweep,
        "stages_ms_per_step": {k: v["ms_per_launch"] * v["launches"] / args.steps for k, v in per_stage.items()},
        "stages": per_stage, "seed_s": t_seed,
    }

    # end to end through the public API with host buffers
    if not args.no_e2e:
        hp = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
        hv = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
        ht = torch.from_numpy(pt.astype(np.int32)).pin_memory()
        sim.read_particles(hp, hv)
        torch.cuda.synchronize()
        barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            sim.set_particles(hp, hv, ht)
            sim.step(dt)
            sim.read_particles(hp, hv, sync=False)
        f1.record(stream)
        barrier()
        ems = max_over_ranks(f0.elapsed_time(f1) / args.steps)
        line["e2e"] = {"value": job_rate(world, ems), "unit": UNIT, "h2d_bytes_per_step": int(n * 28),
                       "d2h_bytes_per_step": int(n * 24),
                       "api": "Simulator.set_particles(pinned host) + step(dt) + read_particles(pinned host)"}

    # standalone solve (128^3, tanh slab + sphere, 1000:1, N(0,1) rhs) to 1e-6
    if not args.no_solve and rank == 0:
        line["solve"] = solve_leg(args)

    # mixed-precision step
    if not args.no_mixed and rank == 0 and args.precision == "fp32":
        sim = None
        torch.cuda.empty_cache()
        line["mixed"] = mixed_leg(args, pos, vel, pt, dt, ms)

    # accuracy of the FP32 and 16-bit-hierarchy steps against the FP64 oracle
    if not args.no_accuracy and rank == 0:
        sim = None
        torch.cuda.empty_cache()
        line["accuracy"] = accuracy_leg(args, pos, vel, pt, dt)

    # differentiable asteroid: gradient of |phi_T - phi*|^2 with respect to v0
    if not args.no_adjoint and rank == 0:
        sim = None
        torch.cuda.empty_cache()
        line["adjoint"] = adjoint_leg(args)

    if not args.no_rt and rank == 0:
        sim = None
        torch.cuda.empty_cache()
        line["rayleigh_taylor"] = rt_leg(args)
        torch.cuda.empty_cache()
        line["rayleigh_taylor"]["gradient"] = rt_grad_leg(args)

    # CPU baseline: the oracle on a bounded sample of the same workload
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        threads = os.cpu_count() or 1
        times = cpu_oracle_steps(cfg, pos, vel, pt, 1, threads)
        line["cpu_baseline"] = {"value": 1.0 / times[0], "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"1 full oracle step of the same {args.res}^3/{args.ppc}ppc dam break "
                                          f"({n:,} particles), all host threads"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ranks.close()
    return 0


def sweep_roofline(sim, ncell, peak, peak_kind, nsweeps=60):
    """The solver's dominant kernel, the finest level's fused red-black sweep
    (k_rb_tile_tma, 28.8% of the step's device time in the ncu launch list),
    timed alone right after the timed region: nsweeps sweeps back to back
    (programmatic dependent launch, as inside a solve) on the step's own last
    hierarchy, with CUDA events on the launching stream.  24 algorithmic bytes
    per cell: read p, b, bx, by, bz, write p (the diagonal is formed from the
    faces)."""
    import torch

    solver = sim.solver
    stream = torch.cuda.current_stream()
    solver._smooth(0, 4)  # warm-up
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    solver._smooth(0, nsweeps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / nsweeps
    ab = 24 * ncell
    ach = ab / (ms * 1e-3) / 1e9
    nx = sim.res[0]
    name = "k_rb_tile_tma<6, 512>" if nx >= 128 else "k_rb_tile_tma<8, 512>" if nx >= 64 else "k_rb_tile_tma"
    return {"kernel": name, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
            "frac": ach / peak, "peak_kind": peak_kind, "algorithmic_bytes_per_launch": ab, "us_per_launch": ms * 1e3,
            "launches_timed": nsweeps, "note": "working set (50 MB) L2-resident between sweeps, as inside a solve"}


def solve_leg(args):
    import torch

    from pfflip import scenes
    from pfflip._arrays import DeviceArray
    from pfflip.poisson import MGPCG

    r = args.res
    bx, by, bz, b, _ = scenes.solve_problem((r, r, r), seed=42)
    dev = lambda a: DeviceArray(torch.from_numpy(a).cuda())  # noqa: E731
    out = {"workload": f"standalone solve {r}^3, 1000:1, tol 1e-6, pre=post=3"}
    ref64 = None
    if not args.no_solve_oracle:
        from oracle import oracle as O

        O.set_threads(os.cpu_count() or 1)
        t0 = time.perf_counter()
        b64 = b.astype(np.float64)
        ref64, it64, rel64 = O.fp64_reference_solve(bx, by, bz, b64, tol=1e-12)
        f64 = [a.astype(np.float64) for a in (bx, by, bz)]
        diag64 = O.compute_diag(*f64)
        out["fp64_oracle"] = {"tol": 1e-12, "iters": it64, "rel": rel64, "cpu_s": time.perf_counter() - t0,
                              "threads": O.get_threads(),
                              "errors": "err_vs_fp64 = max|x - mean(x) - x64| / max|x64| (x64 zero-mean); "
                                        "residual_fp64 = max|b - A x| / max|b| in binary64 (A x = the "
                                        "divergence a projection with x leaves, times -dx/dt)"}
    for var in args.solve_variants.split(","):
        prec, stencil = var.split("_")
        s = MGPCG((r, r, r), "cuda", pre=3, post=3, precision=prec, stencil=stencil, use_graphs=not args.no_graphs)
        s.build_hierarchy(dev(bx), dev(by), dev(bz))
        x = DeviceArray.zeros((r, r, r))
        bd = dev(b)
        s.solve(bd, x, tol=1e-6, max_iter=100)  # warm-up (graph capture)
        ts = []
        for _ in range(args.solve_repeats):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            it, rel = s.solve(bd, x, tol=1e-6, max_iter=100)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        rec = {"ms": float(np.median(ts)), "iters": it, "rel": rel, "converged": rel < 1e-6}
        if ref64 is not None:
            xv = x.numpy().astype(np.float64)
            ax64 = O.apply_A(xv, *f64, diag64, dtype=np.float64, stencil="flux")
            rec["residual_fp64"] = float(np.abs(b64 - ax64).max() / np.abs(b64).max())
            xv -= xv.mean()
            rec["err_vs_fp64"] = float(np.abs(xv - ref64).max() / np.abs(ref64).max())
        out[f"{prec}_{stencil}"] = rec
        del s
    return out


def mixed_leg(args, pos, vel, pt, dt, ms_fp32):
    import torch

    from pfflip import Simulator

    res = {}
    for prec in ("fp16", "bf16"):
        cfg = workload_cfg(args, precision=prec)
        sim = Simulator(cfg)
        sim.set_particles(pos, vel, pt)
        for _ in range(args.warmup):
            sim.step(dt)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        recs = [sim.step(dt) for _ in range(args.steps)]
        e1.record()
        torch.cuda.synchronize()
        m = e0.elapsed_time(e1) / args.steps
        res[prec] = {"ms_per_step": m, "steps_per_s": 1000.0 / m, "speedup_vs_fp32": ms_fp32 / m,
                     "pcg_iter_mean": float(np.mean([r["pcg_iter"] for r in recs]))}
        del sim
        torch.cuda.empty_cache()
    return res


def accuracy_leg(args, pos, vel, pt, dt, warm_steps=2):
    """Errors of one step of the workload against the binary64 oracle, for the
    plain FP32 step and the FP16/BF16-hierarchy steps.

    The particle state after ``warm_steps`` FP32 steps from the seed (so the
    velocities are not zero) is the input of every variant and of the oracle.
    Each variant runs the step's stages on the GPU: sort/P2G, phi/beta,
    u* + gravity, RHS, hierarchy, MG-PCG at the step's tolerance, projection.
    The oracle (pf_oracle.hpp in binary64, 1e-12 CG) is fed the same inputs:

    * phi: binary64 P2G + eq. (7) from the same particles (the hierarchy's
      precision does not reach phi, so one value serves every variant);
    * pressure: the binary64 solve of the GPU's own system (its beta and RHS),
      error after mean removal, relative to max|p64| -- the solver's error;
      and against the all-binary64 pipeline from the particles;
    * divergence: max|div u|/dx after the GPU projection, next to the oracle's
      binary64 projection of the same velocities with p64, and the relative
      error of the projected face velocities."""
    import dataclasses

    import torch

    from oracle import oracle as O
    from pfflip import Simulator

    threads = os.cpu_count() or 1
    O.set_threads(threads)
    t_cpu = 0.0
    cfg32 = workload_cfg(args, precision="fp32")
    sim = Simulator(cfg32)
    sim.set_particles(pos, vel, pt)
    for _ in range(warm_steps):
        sim.step(dt)
    hp, hv, ht = sim.px.numpy(), sim.pv.numpy(), sim.ptype.numpy()
    del sim
    torch.cuda.empty_cache()

    c64 = dataclasses.replace(cfg32, pcg_tol=1e-12, pcg_max_iter=1000)
    t0 = time.perf_counter()
    o = O.OracleSim(c64, dtype=np.float64, nthreads=threads, stencil="flux")
    o.set_particles(hp, hv, ht)
    o._p2g()
    o._phase_field_and_coefficients()
    o._save_vel_star()
    o._add_forces(dt)
    it_pipe, rel_pipe = o._pressure_solve(dt)
    p_pipe = o.pressure - o.pressure.mean()
    phi64 = o.phi_cell.copy()
    t_cpu += time.perf_counter() - t0

    out = {"workload": f"one step of dam_break {args.res}^3 {args.ppc}ppc after {warm_steps} FP32 steps, "
                       f"pcg_tol {args.tol}",
           "oracle": "pf_oracle.hpp binary64, CG to 1e-12", "threads": threads}
    p64 = None
    for prec in ("fp32", "fp16", "bf16"):
        sim = Simulator(workload_cfg(args, precision=prec))
        sim.set_particles(hp, hv, ht)
        sim._p2g()
        sim._phase_field_and_coefficients()
        sim._add_forces(dt, save_vel_star=True)
        it, rel = sim._pressure_solve(dt)
        p = sim.pressure.numpy().astype(np.float64)
        p -= p.mean()
        if p64 is None:  # the GPU's system is the same for every variant: solve it once
            t0 = time.perf_counter()
            beta = [b.numpy().astype(np.float64) for b in sim.beta]
            rhs = sim.rhs.numpy().astype(np.float64)
            p64, it64, rel64 = O.fp64_reference_solve(*beta, rhs, tol=1e-12, max_iter=1000)
            vel_pre = [v.numpy().astype(np.float64) for v in sim.vel]
            o.pressure[...] = p64
            for ax in range(3):
                o.vel[ax][...] = vel_pre[ax]
                o.beta[ax][...] = beta[ax]
            o._project(dt)
            div64 = o._max_divergence()
            vel64 = [v.copy() for v in o.vel]
            t_cpu += time.perf_counter() - t0
            phi = sim.phi_cell.numpy().astype(np.float64)
            out["phi_err_vs_fp64"] = float(np.abs(phi - phi64).max())
            out["phi_note"] = "max|phi - phi64| (phi in [0, 1]); P2G and eq. (7) are FP32 in every variant"
            out["pressure_fp64_system"] = {"iters": it64, "rel": rel64, "max_div_after_projection": div64}
            out["pressure_fp64_pipeline"] = {"iters": it_pipe, "rel": rel_pipe}
        sim._project(dt)
        div = sim._max_divergence()
        vp = [v.numpy().astype(np.float64) for v in sim.vel]
        vscale = max(np.abs(v).max() for v in vel64)
        out[prec] = {
            "pcg_iter": it, "pcg_rel": rel,
            "pressure_err_vs_fp64": float(np.abs(p - p64).max() / np.abs(p64).max()),
            "pressure_err_vs_fp64_pipeline": float(np.abs(p - p_pipe).max() / np.abs(p_pipe).max()),
            "max_div_after_projection": div,
            "velocity_err_vs_fp64_projection": float(max(np.abs(a - b).max() for a, b in zip(vp, vel64)) / vscale),
        }
        del sim
        torch.cuda.empty_cache()
    out["cpu_s"] = t_cpu
    return out


def rt_seed_device(cfg, dev, chunk=1 << 23):
    """Rayleigh-Taylor particles on the device: the jittered lattice tagged by
    reference height (heavy above Ly/2), displaced vertically by the 16 modes
    (scenes.rt_profile) chunk by chunk on the GPU."""
    import torch

    from pfflip import scenes

    pos_ref, ptype, amps, waves = scenes.rayleigh_taylor_lattice(cfg)
    x = torch.from_numpy(pos_ref).to(dev)
    a = torch.tensor(amps, dtype=torch.float64, device=dev)
    for s0 in range(0, x.shape[0], chunk):
        xs = x[s0:s0 + chunk]
        d = scenes.rt_profile(xs.double(), waves, cfg.domain_size, xp=torch) @ a
        xs[:, 1] = (xs[:, 1].double() + d).float()
    return x, ptype, amps, waves


def rt_leg(args):
    """Rayleigh-Taylor: heavy phase (1000) over light (1) across
    y = 0.5 + sum_k a_k cos(2 pi (m_k x + n_k z)), 16 modes with a_k ~ U(0, 0.01)
    and (m_k, n_k) in 1..4 drawn from the seed; 8 ppc.  Steps/s of the plain
    FP32 step and of the 16-bit-hierarchy step at the same fixed dt."""
    import torch

    from pfflip import Config, Simulator

    r = args.rt_res
    base = Config(res=(r, r, r), dx=1.0 / r, ppc=8, seed=42, droplets=False, pcg_tol=args.tol, device="cuda")
    dev = torch.device("cuda")
    t0 = time.perf_counter()
    pos, pt, amps, waves = rt_seed_device(base, dev)
    seed_s = time.perf_counter() - t0
    vel = torch.zeros_like(pos)
    dt = fixed_dt(base.dx)
    out = {"workload": f"rayleigh_taylor {r}^3 8ppc 16 modes", "particles": int(pos.shape[0]), "dt": dt,
           "seed_s": seed_s, "modes": {"a": [float(a) for a in amps], "mn": [[int(m), int(n)] for m, n in waves]}}
    for prec in ("fp32", "fp16"):
        cfg = Config(res=(r, r, r), dx=1.0 / r, ppc=8, seed=42, droplets=False, pcg_tol=args.tol, device="cuda",
                     precision=prec)
        sim = Simulator(cfg)
        sim.set_particles(pos, vel, pt)
        for _ in range(2):
            sim.step(dt)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        recs = [sim.step(dt) for _ in range(max(args.steps // 2, 3))]
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / len(recs)
        out[prec] = {"ms_per_step": ms, "steps_per_s": 1000.0 / ms,
                     "pcg_iter_mean": float(np.mean([x["pcg_iter"] for x in recs])),
                     "max_div": float(recs[-1]["max_div"])}
        del sim
        torch.cuda.empty_cache()
    out["fp16"]["speedup_vs_fp32"] = out["fp32"]["ms_per_step"] / out["fp16"]["ms_per_step"]
    return out


def rt_grad_leg(args):
    """Gradient of the final interface-height variance of the Rayleigh-Taylor
    scene with respect to the 16 mode amplitudes (pfflip.adjoint.
    RTAmplitudeGradient), at --rt-grad-res with --rt-grad-steps steps and
    checkpoints every 5; checked against FP64 central differences of the
    oracle at 32^3 / 20 steps on the two largest components."""
    import torch

    from pfflip import Config
    from pfflip.adjoint import RTAmplitudeGradient

    def cfg_at(r):
        return Config(res=(r, r, r), dx=1.0 / r, ppc=8, seed=42, droplets=False, pcg_tol=1e-6, pcg_max_iter=400,
                      device="cuda")

    r, steps = args.rt_grad_res, args.rt_grad_steps
    cfg = cfg_at(r)
    dt = fixed_dt(cfg.dx)
    g = RTAmplitudeGradient(cfg, dt, steps, checkpoint_every=5, adjoint_tol=1e-6)
    g.gradient()  # warm-up
    a = torch.tensor(g.amps0, dtype=torch.float64, device="cuda", requires_grad=True)
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    torch.cuda.synchronize()
    g.ds.adjoint_solves.clear()
    e0.record()
    loss = g.loss(a)
    e1.record()
    loss.backward()
    e2.record()
    torch.cuda.synchronize()
    out = {"workload": f"rayleigh_taylor {r}^3 8ppc, {steps} steps from rest, checkpoint every 5; "
                       "loss = variance over (x, z) columns of dx * sum_y (1 - phi)",
           "particles": int(g.pos_ref.shape[0]), "dt": dt, "loss": float(loss.detach()),
           "grad_a": a.grad.cpu().numpy().tolist(), "forward_ms": e0.elapsed_time(e1),
           "backward_ms": e1.elapsed_time(e2),
           "adjoint_solve_iters_mean": float(np.mean([it for it, _ in g.ds.adjoint_solves]))}
    del g
    torch.cuda.empty_cache()
    if not args.no_rt_fd:
        from oracle import oracle as O
        from pfflip import scenes

        fr, fsteps = 32, 20
        cf = cfg_at(fr)
        dtf = fixed_dt(cf.dx)
        gs = RTAmplitudeGradient(cf, dtf, fsteps, checkpoint_every=5, adjoint_tol=1e-6)
        _, grad = gs.gradient()
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        comps, unstable = [], []

        def oracle_loss(amps):
            pos = scenes.rt_displace(gs.pos_ref_host, amps, gs.waves, cf.domain_size)
            return O.rt_interface_variance(cf, pos, gs.ptype, dtf, fsteps, nthreads=threads)

        for k in np.argsort(-np.abs(grad))[:4]:
            fd, e, fds = O.stable_central_difference(lambda x: oracle_loss(gs.amps0 + x * np.eye(16)[int(k)]))
            if fd is None:
                unstable.append({"k": int(k), "grad": float(grad[k]), "fd_ladder": fds})
                continue
            comps.append({"k": int(k), "grad": float(grad[k]), "fd": fd, "eps": e, "fd_ladder": fds,
                          "rel_err": abs(grad[k] - fd) / abs(fd)})
            if len(comps) == 2:
                break
        out["fd_check"] = {"res": fr, "steps": fsteps, "oracle": "binary64, solve to 1e-12",
                           "method": "central differences at eps 1e-6, 3e-7, 1e-7, 3e-8, 1e-8; a component is checked "
                                     "at the first two consecutive steps that agree to 2e-4 (away from the jumps "
                                     "that flipping liquid tags and masks put into the loss)",
                           "components": comps, "no_stable_difference": unstable,
                           "max_rel_err": max(c["rel_err"] for c in comps) if comps else None,
                           "cpu_s": time.perf_counter() - t0, "threads": threads}
        del gs
        torch.cuda.empty_cache()
    return out


def adjoint_leg(args):
    """Differentiable asteroid: liquid pool y < 0.3 plus a liquid sphere (r = 0.1
    at (0.5, 0.7, 0.5)) moving with v0 + N(0, 0.01^2) perturbations, 8 ppc; loss
    |phi_T - phi*|^2 with phi* from a run with v0 = (0.5, -2, 0); gradient with
    respect to v0 through the adjoint kernels, checkpoint every 5 steps."""
    import dataclasses

    import torch

    from pfflip import Config, scenes
    from pfflip.adjoint import DiffSim

    steps, every = args.adjoint_steps, 5

    def setup(r):
        cfg = Config(res=(r, r, r), dx=1.0 / r, ppc=8, seed=42, droplets=False, pcg_tol=1e-6, pcg_max_iter=400,
                     device="cuda")
        pos, vel, pt, sphere, pert = scenes.asteroid_pool(cfg, v0=(0.0, -2.0, 0.0))
        base = np.zeros_like(vel)
        base[sphere] = pert[sphere]
        return cfg, 0.25 * cfg.dx / 2.5, pos, pt, sphere, base

    def gpu_grad(cfg, dt, pos, pt, sphere, base, timed):
        ds = DiffSim(cfg, pt, dt, checkpoint_every=every, adjoint_tol=1e-6)
        dev = torch.device("cuda")
        x0 = torch.from_numpy(pos).to(dev)
        b0 = torch.from_numpy(base).to(dev)
        mask = torch.from_numpy(sphere).to(dev)[:, None].float()
        with torch.no_grad():
            vt = b0 + mask * torch.tensor([0.5, -2.0, 0.0], device=dev)[None, :]
            phi_star = ds.phase_field(ds.rollout(x0, vt, steps)[0]).double()

        def run():
            v0 = torch.tensor([0.0, -2.0, 0.0], device=dev, requires_grad=True)
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            torch.cuda.synchronize()
            e0.record()
            xT, _ = ds.rollout(x0, b0 + mask * v0[None, :], steps)
            loss = ((ds.phase_field(xT).double() - phi_star) ** 2).sum()
            e1.record()
            loss.backward()
            e2.record()
            torch.cuda.synchronize()
            return float(loss.detach()), v0.grad.double().cpu().numpy(), e0.elapsed_time(e1), e1.elapsed_time(e2)

        if timed:
            run()  # warm-up
        ds.adjoint_solves.clear()
        out = run()
        solves = list(ds.adjoint_solves)
        phs = phi_star.cpu().numpy()
        del ds
        torch.cuda.empty_cache()
        return out, solves, phs

    r = args.adjoint_res
    cfg, dt, pos, pt, sphere, base = setup(r)
    (loss, grad, fwd_ms, bwd_ms), solves, phs = gpu_grad(cfg, dt, pos, pt, sphere, base, True)
    out = {"workload": f"differentiable asteroid {r}^3 8ppc, {steps} steps, checkpoint every {every}",
           "particles": int(len(pos)), "dt": dt, "loss": loss, "grad_v0": grad.tolist(),
           "forward_ms": fwd_ms, "backward_ms": bwd_ms, "forward_ms_per_step": fwd_ms / steps,
           "backward_ms_per_step": bwd_ms / steps,
           "adjoint_solve_iters_mean": float(np.mean([it for it, _ in solves])),
           "adjoint_solve_rel_max": float(max(rel for _, rel in solves))}
    if not args.no_adjoint_fd:
        from oracle import oracle as O

        fr = args.adjoint_fd_res or r
        if fr != r:
            cfg, dt, pos, pt, sphere, base = setup(fr)
            (_, grad, _, _), _, phs = gpu_grad(cfg, dt, pos, pt, sphere, base, False)
        threads = os.cpu_count() or 1
        c64 = dataclasses.replace(cfg, pcg_tol=1e-12, pcg_max_iter=1000)

        def fd_loss(v):
            vv = base.astype(np.float64)
            vv[sphere] += v
            sim = O.OracleSim(c64, dtype=np.float64, nthreads=threads, stencil="flux")
            sim.set_particles(pos, vv, pt)
            for _ in range(steps):
                sim.step(dt)
            sim._p2g()
            sim._phase_field_and_coefficients()
            return float(((sim.phi_cell - phs) ** 2).sum())

        eps = 1e-6
        v = np.array([0.0, -2.0, 0.0])
        t0 = time.perf_counter()
        fd = np.array([(fd_loss(v + eps * e) - fd_loss(v - eps * e)) / (2 * eps) for e in np.eye(3)])
        out["fd_check"] = {"res": fr, "grad_v0": grad.tolist(), "fd_grad_v0": fd.tolist(), "eps": eps,
                           "oracle": "binary64, solve to 1e-12",
                           "max_rel_err": float(np.abs(grad - fd).max() / np.abs(fd).max()),
                           "cpu_s": time.perf_counter() - t0, "threads": threads}
    return out


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.rt_only:
        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        rt = rt_leg(args)
        rt["gradient"] = rt_grad_leg(args)
        print(json.dumps({"rayleigh_taylor": rt}), flush=True)
        return 0
    if args.adjoint_only:
        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps({"adjoint": adjoint_leg(args)}), flush=True)
        return 0
    if args.solve_only:
        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps({"solve": solve_leg(args)}), flush=True)
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
