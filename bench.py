"""Benchmark of the fused thermal LBM time step on B200.

Workload (default): the 3D differentially heated cubic cavity, D3Q19 MRT +
D3Q7 thermal, 128^3 nodes on a tanh-stretched grid (factor 1.5) on every axis,
Ra = 1e5, Pr = 0.71, Ma = 0.1, rest initial state (rho = 1, u = 0, T = 0),
FP64 storage and arithmetic (the drop-in).  A bench "step" is `--inner` LBM
iterations (one lbm_step call).  Inputs are synthetic: the reference ships no
data and none is needed.

value  MLUPS of the fused step kernel with the state resident in HBM, timed
       with CUDA events on the library's stream (the state, 2 x 436 MB
       ping-pong, is larger than the 126 MB L2, so no flush is needed);
e2e    the same metric through the public C ABI with host buffers: every step
       uploads the initial macroscopic fields from pinned host memory
       (lbm_init_equilibrium), runs the iterations and reads the fields back
       (lbm_get_macro);
roofline  algorithmic bytes per lattice update (2*Q*b_pop + 2*b_aux: 432 B in
       FP64 3D) x nodes / mean kernel duration, against the measured HBM copy
       bandwidth;
cpu_baseline  the CPU restatement of the reference (C, OpenMP) on this host's
       cores, on a bounded sample of the same workload.

`--impl reference` times the reference's CPU algorithm instead: the Fortran
reference cannot be compiled here (no Fortran compiler, no MPI), so its C
restatement runs on all host cores, one full-domain iteration per step.
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

WORKLOADS = {
    # name: (dim, nx, ny, nz, grid, stretch, Ra, Pr)
    "cavity3d_128": (3, 128, 128, 128, "tanh", 1.5, 1e5, 0.71),
    "cavity2d_2048": (2, 2048, 2048, 1, "tanh", 1.5, 1e6, 0.71),
    "cavity2d_128": (2, 128, 128, 1, "tanh", 1.5, 1e4, 0.71),
}
BYTES_PER_VALUE = {"f64": 8, "f32": 4}
AUX_BYTES = {"f64": 8, "f32": 4}


def bytes_per_lup(dim: int, storage: str) -> int:
    q = 14 if dim == 2 else 26
    return 2 * q * BYTES_PER_VALUE[storage] + 2 * AUX_BYTES[storage]


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(workload: str, storage: str):
    """Per-launch DRAM bytes of the step kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        parts = line.split()
        if len(parts) >= 3 and parts[0] == workload and parts[1] == storage:
            try:
                return float(parts[2])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: str | None):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.gpu is not None:
            cmd += ["-i", self.gpu]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self._t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for name, flag in zip(names, p[5:9]):
                if flag.lower() in ("active", "1"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_sample(wl, seconds: float = 12.0, max_steps: int = 200):
    """Time the oracle (C restatement of the reference, OpenMP) on this host."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    dim, nx, ny, nz, grid, stretch, Ra, Pr = wl
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    o = oracle.Oracle(dim, nx, ny, nz, grid=grid, stretch=stretch, Ra=Ra, Pr=Pr)
    shape = o.shape
    one, zero = np.ones(shape), np.zeros(shape)
    o.set_macro(one, zero, zero, zero if dim == 3 else None, zero)
    o.step(1)
    steps, t0 = 0, time.perf_counter()
    while steps < max_steps:
        o.step(1)
        steps += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    nn = nx * ny * nz
    return {"value": nn * steps / dt / 1e6, "unit": "MLUPS", "cores": oracle.get_threads(), "kind": "port",
            "sample": f"{steps} full-domain iterations of {nx}x{ny}x{nz} (FP64, C restatement, "
                      f"{oracle.get_threads()} OpenMP threads), {dt:.1f} s"}


def cpu_sample_batch(seconds: float = 12.0, max_rounds: int = 200, warmup: int = 1):
    """Time the oracle (C restatement of the reference, OpenMP) on the first 8
    cavities of the seed-0 batch sweep, one iteration of each per round."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from __graft_entry__ import load_package
    pkg = load_package()
    oracle.set_threads(os.cpu_count() or 1)
    specs = pkg.sweep_specs(256, seed=0)[:8]
    orc = []
    for sp in specs:
        m = sp["coords"]
        orc.append(oracle.Oracle(2, sp["nx"], sp["ny"], 1, x=m.x, y=m.y, dt=m.dt, length_LB=m.length_LB,
                                 Ra=sp["Ra"], Pr=sp["Pr"]))
    for _ in range(warmup):
        for o in orc:
            o.step(1)
    rounds, t0 = 0, time.perf_counter()
    while rounds < max_rounds:
        for o in orc:
            o.step(1)
        rounds += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    nodes = sum(sp["nx"] * sp["ny"] for sp in specs)
    return {"value": nodes * rounds / dt / 1e6, "unit": "MLUPS", "cores": oracle.get_threads(), "kind": "port",
            "sample": f"{rounds} iterations of the first 8 sweep cavities ({nodes} nodes; FP64, C restatement, "
                      f"{oracle.get_threads()} OpenMP threads), {dt:.1f} s", "rounds": rounds, "seconds": dt,
            "nodes": nodes}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=None)
    return world, rank, local


def run_reference_batch(args):
    """batch256 on the CPU: the C restatement advances the first cavities of
    the same seeded sweep, one iteration of each per step (a bounded sample)."""
    c = cpu_sample_batch(seconds=float("inf"), max_rounds=args.steps, warmup=args.warmup)
    nodes, dt, v = c["nodes"], c["seconds"], c["value"]
    line = {"impl": "reference", "metric": "MLUPS", "value": v, "unit": "MLUPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "batch256", "sample": "first 8 cavities of the seed-0 sweep, one iteration each "
                                                         "per step", "nodes": nodes},
            "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": c["cores"], "kind": "port",
                             "sample": f"{args.steps} iterations of 8 sweep cavities ({nodes} nodes)"},
            "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference(args, world, rank):
    if rank != 0:
        return
    if args.workload == "batch256":
        return run_reference_batch(args)
    if args.workload == "unet":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no network: the warm-start "
                          "surrogate has no counterpart to time"}), flush=True)
        return
    if args.workload == "steady":
        print(json.dumps({"impl": "reference", "unavailable": "time to a steady state of the CPU restatement is "
                          "hours at these sizes (10^5-10^6 iterations per cavity); its per-iteration rate is the "
                          "reference arm of the cavity workloads"}), flush=True)
        return
    wl = WORKLOADS[args.workload]
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    dim, nx, ny, nz, grid, stretch, Ra, Pr = wl
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    o = oracle.Oracle(dim, nx, ny, nz, grid=grid, stretch=stretch, Ra=Ra, Pr=Pr)
    shape = o.shape
    one, zero = np.ones(shape), np.zeros(shape)
    o.set_macro(one, zero, zero, zero if dim == 3 else None, zero)
    for _ in range(args.warmup):
        o.step(1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.step(1)
    dt = time.perf_counter() - t0
    nn = nx * ny * nz
    v = nn * args.steps / dt / 1e6
    line = {
        "impl": "reference", "metric": "MLUPS", "value": v, "unit": "MLUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": config_of(args, wl), "iterations_per_step": 1,
        "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": oracle.get_threads(), "kind": "port",
                         "sample": f"{args.steps} full-domain iterations per run, one per step; the Fortran "
                                   f"reference is not compilable here (no Fortran compiler / MPI), its C "
                                   f"restatement runs instead"},
        "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_of(args, wl):
    """The workload, identical in both arms (the metric is per lattice update,
    so how many iterations one bench step runs is not part of it)."""
    dim, nx, ny, nz, grid, stretch, Ra, Pr = wl
    return {"workload": args.workload, "lattice": "D2Q9+D2Q5" if dim == 2 else "D3Q19+D3Q7",
            "nodes": [nx, ny, nz] if dim == 3 else [nx, ny], "grid": f"{grid} stretch {stretch}",
            "Ra": Ra, "Pr": Pr, "Ma": 0.1, "storage": args.storage, "mode": args.mode,
            "init": "rest (rho=1, u=0, T=0)",
            "l2": "state larger than L2 (2 x ping-pong buffers), no flush",
            "parallelism": f"{args.gpus} independent cavities, one per GPU"}


def kernel_config(cav, pkg):
    """How this arm runs the workload (not part of the workload itself)."""
    kc = {"kernel": cav.kernel}
    if cav.kernel == "march":
        kc["march_blocks"] = cav.get_option(pkg.lbm.OPT_NBLOCKS)
        kc["l2_promotion"] = ["none", "64B", "128B", "256B"][cav.get_option(pkg.lbm.OPT_L2PROMO)]
        if cav.dim == 3:
            kc["tile_rows"] = cav.get_option(pkg.lbm.OPT_TILEY)
            kc["plan"] = ["z-lockstep, balanced tails", "contiguous shares"][cav.get_option(pkg.lbm.OPT_PLAN)]
    return kc


def _reduce(x: float, world: int, op: str) -> float:
    """max / sum of a host scalar over ranks (NCCL; identity on one rank)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def _barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_batch(args, world, rank, local):
    """The seeded sweep of 256 2D cavities (widths 64..512, aspect 1-4, Ra
    1e3..1e6, Pr 0.71..7, tanh stretch 1..2) through one persistent kernel per
    step, against stepping each cavity with its own launch (same precision).
    On N ranks each rank advances its own seeded sweep (seed = rank: weak
    scaling), or with --batch-shard one sweep split by LPT over node counts
    (strong scaling); no data crosses ranks while stepping."""
    import torch
    torch.cuda.set_device(local)
    from __graft_entry__ import load_package
    pkg = load_package()
    ns = args.sweep  # all 256, or the first few for a profile
    if args.batch_shard:
        all_specs = pkg.sweep_specs(256, seed=0)[:ns]
        idx, specs = pkg.sharding.my_share(all_specs, world, rank)
        n_total, scaling = len(all_specs), "strong"
    else:
        specs = pkg.sweep_specs(256, seed=rank)[:ns]
        idx, n_total, scaling = list(range(rank * ns, rank * ns + ns)), ns * world, "weak"
    b = pkg.Batch(2, specs, storage=args.storage, mode=args.mode, device=local)
    b.initial()
    if args.tile:
        b.set_option("tile", args.tile)
        tuned = {"tile": args.tile, "nblocks": b.get_option("nblocks")}
    else:
        tuned = b.tune(steps=6)
    stream = torch.cuda.ExternalStream(b.stream_ptr(), device=torch.device("cuda", local))

    def timed(nsteps, reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        _barrier(world)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            b.step(nsteps)
        e1.record(stream)
        torch.cuda.synchronize()
        _barrier(world)
        return _reduce(e0.elapsed_time(e1), world, "max")

    for _ in range(args.warmup):
        b.step(args.inner)
    b.synchronize()
    sampler = None
    if not args.no_clocks and rank == 0:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        sampler = ClockSampler(vis.split(",")[local] if vis else str(local))
        sampler.start()
        time.sleep(0.3)
    l0 = pkg.kernel_launches()
    ms = timed(args.inner, args.steps)
    launches = pkg.kernel_launches() - l0
    clocks = sampler.stop() if sampler else None
    nodes = b.nodes
    nodes_all = _reduce(float(nodes), world, "sum")
    iters = args.steps * args.inner
    value = nodes_all * iters / (ms / 1e3) / 1e6
    # one launch per cavity per step, same batch and precision
    b.set_option("persistent", 0)
    b.step(2)
    base_steps = max(2, args.inner // 10)
    ms_base = timed(base_steps, 2)
    baseline = nodes_all * base_steps * 2 / (ms_base / 1e3) / 1e6
    b.set_option("persistent", 1)
    bpl = bytes_per_lup(2, args.storage)
    peak, peak_kind = measured_peak()
    achieved = bpl * nodes * iters / (ms / 1e3) / 1e9
    e2e = None
    if not args.no_e2e:
        # every step: upload each member's initial fields from pinned memory,
        # advance, read back each member's Nusselt numbers
        big = max(m.nnode for m in b.members)
        pin = {k: torch.zeros(big, dtype=torch.float64, pin_memory=True).numpy() for k in ("rho", "u", "v", "T")}
        pin["rho"][:] = 1.0
        reps = max(1, args.steps // 4)
        _barrier(world)
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(reps):
            for m in b.members:
                nn = m.nnode
                m.init_equilibrium(*(pin[k][:nn].reshape(m.shape) for k in ("rho", "u", "v")), None,
                                   pin["T"][:nn].reshape(m.shape))
            b.step(args.inner)
            nu_hot, _ = b.nusselt()
        f1.record(stream)
        torch.cuda.synchronize()
        _barrier(world)
        ems = _reduce(f0.elapsed_time(f1), world, "max")
        e2e = {"value": nodes_all * args.inner * reps / (ems / 1e3) / 1e6, "unit": "MLUPS",
               "h2d_bytes_per_step": 4 * nodes * 8, "d2h_bytes_per_step": 2 * 8 * len(specs),
               "path": "lbm_init_equilibrium per member (pinned host fields) + lbm_batch_step + lbm_batch_nusselt"}
        # the one collective of the data path: every cavity's result to every rank
        got = pkg.sharding.gather_by_index(idx, {"nu_hot": nu_hot}, n_total)
        e2e["nusselt_gathered"] = int(np.isfinite(got["nu_hot"]).sum())
    # the C restatement on this host's cores, after the GPU timing: the first 8 sweep cavities
    cpu = cpu_sample_batch() if rank == 0 and world == 1 and not args.no_cpu else None
    if rank == 0:
        line = {
            "metric": "MLUPS", "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": scaling,
            "vs_baseline": None, "dtype": args.storage, "data": "synthetic",
            "config": {"workload": "batch256" if ns == 256 else f"batch256 (first {ns})", "cavities": n_total, "nodes": int(nodes_all), "lattice": "D2Q9+D2Q5",
                       "sweep": "widths {64..512}, aspect 1-4, Ra 1e3-1e6 log, Pr 0.71-7, tanh stretch 1-2, "
                                + ("seed 0 split over ranks by LPT" if args.batch_shard else "seed = rank"),
                       "storage": args.storage, "mode": args.mode, "iterations_per_step": args.inner,
                       "tile": tuned["tile"], "blocks": tuned["nblocks"], "graphs": True,
                       "l2": "state larger than L2 (%.1f GB per GPU)" % (nodes * bpl / 2 / 1e9),
                       "one_launch_per_cavity_mlups": baseline,
                       "speedup_vs_one_launch_per_cavity": value / baseline if baseline else None},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_kind": peak_kind, "bytes_per_lup": bpl, "kernel": "k_march2d_batch"},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    b.close()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


MODEL_PATH = os.path.join(ROOT, "mpi-multi-process-version_b200", "warmstart_unet.npz")


def steady_cold_arm(pkg, cases, max_steps, device):
    """The FP64 drop-in's time to solution: each case from the conduction
    state, one cavity at a time, to the reference's criterion (errorU, errorT
    <= float32(1e-6) at a check every 2000 iterations, 2M:307)."""
    W = pkg.warmstart
    steps, nu, t = [], [], 0.0
    for c in cases:
        cav = pkg.Cavity(2, c["nx"], c["ny"], Ra=c["Ra"], Pr=c["Pr"], coords=c["coords"], storage="f64",
                         device=device)
        cav.initial()
        cav.synchronize()
        t0 = time.perf_counter()
        n, _, _ = cav.run(max_steps, 2000, W.F32_EPS)
        cav.synchronize()
        t += time.perf_counter() - t0
        steps.append(n)
        nu.append(cav.nusselt()[0])
        cav.close()
    return steps, nu, t


def _tau_delta(text):
    """'TAU,DELTA' -> (float, int); 'off' -> None."""
    if text.strip().lower() == "off":
        return None
    tau, delta = text.split(",")
    return float(tau), int(delta)


def time_to_steady(pkg, ncases, max_steps, device, extrapolate=None):
    """Both arms of the time-to-steady comparison on the first `ncases`
    held-out cavities, timed here: FP64 cold one cavity at a time against
    mixed precision (member by member, FP32 to 1e-5 then FP64) + one batch +
    the learned warm start; the Nusselt agreement between them."""
    W = pkg.warmstart
    model = W.WarmStart.load(MODEL_PATH, device=device)
    cases = W.sample_cases(200, seed=2000)[:ncases]
    steps_cold, nu_cold, t_cold = steady_cold_arm(pkg, cases, max_steps, device)
    r = W.solve(cases, init="warm", model=model, storage="auto", max_steps=max_steps, device=device,
                extrapolate=extrapolate)
    nu_cold = np.asarray(nu_cold)
    err = np.abs(np.asarray(r["nu_hot"]) - nu_cold) / np.abs(nu_cold)
    conv = np.asarray(r["status"]) == 1
    return {"cases": ncases, "sides": "128..256", "criterion": "errorU, errorT <= float32(1e-6) every 2000 "
            "iterations", "max_steps": max_steps, "fp64_cold_seconds": t_cold, "warm_batched_seconds": r["seconds"],
            "speedup": t_cold / r["seconds"], "fp64_cold_steps": int(np.sum(steps_cold)),
            "fp64_cold_converged": int(np.sum(np.asarray(steps_cold) < max_steps)),
            "warm_batched_steps": int(np.sum(r["steps"])), "converged_warm_batched": int(conv.sum()),
            "nu_within_1e-4_of_fp64": int((conv & (err <= 1e-4)).sum()), "max_nu_rel_err": float(err.max()),
            "fallbacks": int(np.sum(r["fallback"])), "storage_chosen": r["tuned"]["chosen"],
            "tuned_mlups": {k: r["tuned"][k]["mlups"] for k in ("f64", "f32")},
            # what the run applied: null when off, or when the autotuner chose the mixed run (no extrapolation)
            "extrapolate": None if r.get("extrapolation_factors") is None else
            {"tau": extrapolate[0], "delta": extrapolate[1],
             "members_extrapolated": int(np.sum(np.asarray(r["extrapolation_factors"]) > 0))},
            "arms": "FP64 from the conduction state, one cavity per launch vs. one persistent batch + learned "
                    "warm start + storage chosen by the autotuner (mixed precision member by member if FP32 "
                    "stepping pays for its hand-over, else FP64) + one extrapolation of each member's slowest "
                    "mode (see `extrapolate`, null when off); prediction, tuning, initialisation and the "
                    "extrapolation's host round trips timed"}


def run_unet(args, world, rank, local):
    """The warm-start network's training step on the library's own kernels:
    forward, MSE loss, backward and Adam of the 4-level U-Net (1.95 M
    parameters, bf16 activations, FP32 accumulation) on a batch of 16
    128 x 128 images (seeded random inputs and targets), with the 3x3
    convolutions on the chosen tensor-core path (--tensor-path 0: mma.sync,
    1: tcgen05 with the accumulator in tensor memory).  roofline: the 3x3
    convolutions' FLOPs (forward, data and weight gradients) per step against
    the measured bf16 GEMM peak."""
    import torch
    torch.cuda.set_device(local)
    from __graft_entry__ import load_package
    pkg = load_package()
    S = pkg.surrogate
    S.set_tensor_path(args.tensor_path)
    R, B = 128, 16
    net = S.Net(R=R, device=local, seed=0)
    g = torch.Generator(device="cpu").manual_seed(0)
    x = (torch.randn(B, R, R, S.IN_CH, generator=g) * 0.5).to(torch.bfloat16).cuda(local)
    y = (torch.randn(B * R * R, S.OUT_CH, generator=g) * 0.1).cuda(local)
    stream = net.stream

    def step():
        net.forward(x, B)
        net.loss(y, B)
        net.backward(B)
        net.adam(1e-4)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = pkg.kernel_launches()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    launches = pkg.kernel_launches() - l0
    ms = e0.elapsed_time(e1) / args.steps
    res = {"e1": R, "e2": R // 2, "e3": R // 4, "b": R // 8, "d3": R // 4, "d2": R // 2, "d1": R}
    flops = sum(2.0 * B * res[n[:-1]] ** 2 * 9 * ci * co for n, ci, co in S.layer_table()) * 3
    peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peak, kind = float(json.load(fh)["bf16_tflops"]), "measured"
    except Exception:
        peak, kind = 1590.0, "fallback"
    tflops = flops / (ms * 1e-3) / 1e12
    if rank == 0:
        print(json.dumps({
            "metric": "unet_train_step_ms", "value": ms, "unit": "ms", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16 (FP32 accumulation)", "data": "synthetic",
            "config": {"workload": "unet", "batch": B, "image": R, "params": int(net.n_params),
                       "tensor_path": ["mma.sync", "tcgen05"][args.tensor_path]},
            "roofline": {"bound": "tensor", "achieved": tflops, "peak": peak, "unit": "TFLOP/s",
                         "frac": tflops / peak, "traffic": None, "peak_kind": kind,
                         "flops_per_step": flops, "kernel": "3x3 convolutions (fwd, dgrad, wgrad)"},
            "gpu_launches": launches, "timeouts": S.timeouts(reset=True)}), flush=True)


def run_steady(args, world, rank, local):
    """Time to a steady state on held-out cavities (square, sides 128..256,
    Ra 1e3..1e6 log-uniform, Pr 0.71..7, tanh stretch 1..2; the first
    --cases of the held-out seed the warm-start model never saw): the FP64
    drop-in from the conduction state, one cavity per launch, against mixed
    precision (FP32 storage to residual 1e-5, then FP64) + one persistent
    batch + the learned warm start.  Both run to the
    reference's stop criterion (errorU, errorT <= 1e-6 at a check every 2000
    iterations, 2M:307); the metric is the mixed arm's wall time for all
    cases (lower is better), with the Nusselt agreement between the arms.
    On N ranks the cases are split by LPT over node counts."""
    import torch
    torch.cuda.set_device(local)
    from __graft_entry__ import load_package
    pkg = load_package()
    W = pkg.warmstart
    model = W.WarmStart.load(MODEL_PATH, device=local)
    all_cases = W.sample_cases(200, seed=2000)[:args.cases]
    idx, cases = pkg.sharding.my_share(all_cases, world, rank)
    max_steps = args.max_steps
    steps_cold, nu_cold, t_cold = steady_cold_arm(pkg, cases, max_steps, local)
    # mixed: FP32 storage, one batch, warm start (prediction time included)
    sampler = None
    if not args.no_clocks and rank == 0:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        sampler = ClockSampler(vis.split(",")[local] if vis else str(local))
        sampler.start()
        time.sleep(0.3)
    l0 = pkg.kernel_launches()
    _barrier(world)
    r = W.solve(cases, init="warm", model=model, storage=args.steady_storage, max_steps=max_steps, device=local,
                extrapolate=args.steady_extrapolate)
    launches = pkg.kernel_launches() - l0
    clocks = sampler.stop() if sampler else None
    t_mixed = _reduce(r["seconds"], world, "max")  # prediction and initialisation included
    t_cold = _reduce(t_cold, world, "max")
    got = pkg.sharding.gather_by_index(idx, {"steps_cold": steps_cold, "nu_cold": nu_cold, "steps_mixed": r["steps"],
                                             "nu_mixed": r["nu_hot"], "status": r["status"],
                                             "nodes": [c["nx"] * c["ny"] for c in cases]}, len(all_cases))
    if rank == 0:
        err = np.abs(got["nu_mixed"] - got["nu_cold"]) / np.abs(got["nu_cold"])
        conv = got["status"] == 1
        chosen = (r["tuned"] or {}).get("chosen", args.steady_storage)
        lups = float(np.sum(got["steps_mixed"] * got["nodes"]))
        # algorithmic bytes of the warm arm: FP64 steps at 240 B per update, FP32
        # steps (the transient of a mixed run, or an FP32 run) at 120 B
        low = r.get("steps_low_precision")
        if chosen == "f32":
            nbytes = bytes_per_lup(2, "f32") * lups
        elif low is not None and rank == 0 and world == 1:
            lo = np.asarray(low, dtype=np.float64) * np.asarray([c["nx"] * c["ny"] for c in cases])
            nbytes = bytes_per_lup(2, "f64") * (lups - lo.sum()) + bytes_per_lup(2, "f32") * lo.sum()
        else:
            nbytes = bytes_per_lup(2, "f64") * lups
        bpl = nbytes / lups if lups else 0.0
        peak, peak_kind = measured_peak()
        achieved = nbytes / t_mixed / 1e9
        line = {
            "metric": "time_to_steady_s", "value": t_mixed, "unit": "s", "n_gpus": world, "steps": 1, "warmup": 0,
            "ms_per_step": t_mixed * 1e3, "higher_is_better": False, "scaling": "strong", "vs_baseline": None,
            "dtype": f"storage policy {args.steady_storage} (FP64 residual / Nu sums)", "data": "synthetic",
            "config": {"workload": "steady", "cases": len(all_cases), "sides": "128..256", "criterion":
                       "errorU, errorT <= float32(1e-6) every 2000 iterations", "max_steps": max_steps,
                       "model": os.path.basename(MODEL_PATH), "baseline_arm": "FP64, conduction start, one cavity "
                       "per launch"},
            "time_to_steady": {"fp64_cold_seconds": t_cold, "warm_batched_seconds": t_mixed,
                               "speedup": t_cold / t_mixed, "fp64_cold_steps": int(got["steps_cold"].sum()),
                               "warm_batched_steps": int(got["steps_mixed"].sum()),
                               "converged_warm_batched": int(conv.sum()),
                               "storage_chosen": (r["tuned"] or {}).get("chosen", args.steady_storage),
                               "nu_within_1e-4_of_fp64": int((conv & (err <= 1e-4)).sum()),
                               "max_nu_rel_err": float(err.max()), "fallbacks": int(np.sum(r["fallback"])),
                               "extrapolate": (args.steady_extrapolate
                                               if r.get("extrapolation_factors") is not None else None)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_kind": peak_kind, "bytes_per_lup": bpl,
                         "kernel": "k_march2d_batch, the warm arm's algorithmic bytes (240 B per FP64 update, "
                                   "120 B per FP32 update) over its wall time incl. prediction and host checks"},
            "cpu_baseline": None,
            "e2e": {"value": t_mixed, "unit": "s", "h2d_bytes_per_step": int(4 * 8 * got["nodes"].sum()),
                    "d2h_bytes_per_step": 16 * len(all_cases),
                    "path": "host prediction + lbm_init_warm per member + lbm_batch_run_masked + lbm_batch_nusselt"},
            "gpu_launches": launches, "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--inner", type=int, default=100, help="LBM iterations per bench step")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cavity3d_128",
                    choices=sorted(WORKLOADS) + ["batch256", "steady", "unet"])
    ap.add_argument("--tensor-path", type=int, default=0, choices=[0, 1], help="unet: 0 mma.sync, 1 tcgen05")
    ap.add_argument("--cases", type=int, default=16, help="steady: held-out cavities")
    ap.add_argument("--steady-cases", type=int, default=16,
                    help="cavity workloads: held-out cavities of the time_to_steady object (0: leave it out)")
    ap.add_argument("--steady-storage", default="auto", choices=["auto", "mixed", "f64", "f32"],
                    help="steady workload: storage policy of the warm-started batch")
    ap.add_argument("--steady-extrapolate", type=_tau_delta, default=(3e-5, 10000), metavar="TAU,DELTA|off",
                    help="steady workload and time_to_steady: one extrapolation of each member's slowest mode at "
                         "residual TAU from states DELTA iterations apart (default 3e-5,10000; 'off' to run "
                         "without it)")
    ap.add_argument("--steady-max-steps", type=int, default=3_000_000,
                    help="time_to_steady: iteration cap per cavity, high enough for every case of both arms")
    ap.add_argument("--max-steps", type=int, default=1_500_000, help="steady: iteration cap per cavity")
    ap.add_argument("--storage", default="f64", choices=["f64", "f32"])
    ap.add_argument("--mode", default="fast", choices=["fast", "exact"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-clocks", action="store_true")
    ap.add_argument("--kernel", default="auto", choices=["auto", "direct", "march"])
    ap.add_argument("--nblocks", type=int, default=0, help="persistent blocks of the march kernel (0 = auto)")
    ap.add_argument("--l2promo", type=int, default=-1, help="TMA L2 promotion 0..3 (-1 = library default)")
    ap.add_argument("--tiley", type=int, default=0, help="3D march tile rows 4 or 8 (0 = library default)")
    ap.add_argument("--plan", type=int, default=-1, help="3D march work plan 0 or 1 (-1 = library default)")
    ap.add_argument("--sweep", type=int, default=256, help="batch256: the first N cavities of the sweep (a profile)")
    ap.add_argument("--tile", type=int, default=0, help="batch256: tile width 32/64/128 instead of the autotuner")
    ap.add_argument("--batch-shard", action="store_true",
                    help="batch256 on N GPUs: split one sweep by LPT (strong scaling) instead of one sweep per rank")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        # rank 0 alone times the CPU algorithm; other ranks exit without work
        # and without a process group
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    world, rank, local = dist_setup()
    if args.workload == "batch256":
        return run_batch(args, world, rank, local)
    if args.workload == "steady":
        return run_steady(args, world, rank, local)
    if args.workload == "unet":
        return run_unet(args, world, rank, local)

    import torch
    torch.cuda.set_device(local)
    from __graft_entry__ import load_package
    pkg = load_package()
    wl = WORKLOADS[args.workload]
    dim, nx, ny, nz, grid, stretch, Ra, Pr = wl
    cav = pkg.Cavity(dim, nx, ny, nz, Ra=Ra, Pr=Pr, grid=grid, stretch=stretch, storage=args.storage,
                     mode=args.mode, device=local, kernel=args.kernel, nblocks=args.nblocks)
    if args.l2promo >= 0:
        cav.set_option(pkg.lbm.OPT_L2PROMO, args.l2promo)
    if args.tiley and dim == 3:
        cav.set_option(pkg.lbm.OPT_TILEY, args.tiley)
    if args.plan >= 0 and dim == 3:
        cav.set_option(pkg.lbm.OPT_PLAN, args.plan)
    shape = cav.shape
    # pinned host fields for the end-to-end leg
    pin = {k: torch.zeros(shape, dtype=torch.float64, pin_memory=True) for k in ("rho", "u", "v", "w", "T")}
    pin["rho"].fill_(1.0)
    hostf = {k: t.numpy() for k, t in pin.items()}
    cav.init_equilibrium(hostf["rho"], hostf["u"], hostf["v"], hostf["w"] if dim == 3 else None, hostf["T"])
    stream = torch.cuda.ExternalStream(cav.stream_ptr(), device=torch.device("cuda", local))

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    for _ in range(args.warmup):
        cav.step(args.inner)
    cav.synchronize()

    clocks = None
    sampler = None
    if not args.no_clocks and rank == 0:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        gpu = vis.split(",")[local] if vis else str(local)
        sampler = ClockSampler(gpu)
        sampler.start()
        time.sleep(0.3)

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = pkg.kernel_launches()
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        cav.step(args.inner)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    launches = pkg.kernel_launches() - launches0
    ms = max_over_ranks(e0.elapsed_time(e1))
    if sampler is not None:
        clocks = sampler.stop()

    nn = cav.nnode
    iters = args.steps * args.inner
    value = world * nn * iters / (ms / 1e3) / 1e6
    bpl = bytes_per_lup(dim, args.storage)
    peak, peak_kind = measured_peak()
    ms_launch = ms / iters
    achieved = bpl * nn / (ms_launch / 1e3) / 1e9
    traffic = ncu_traffic(args.workload, args.storage)

    # end-to-end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        h2d = 0
        d2h = 0
        pout = {k: torch.zeros(shape, dtype=torch.float64, pin_memory=True).numpy()
                for k in ("rho", "u", "v", "w", "T")}
        nfield = 5 if dim == 3 else 4
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            cav.init_equilibrium(hostf["rho"], hostf["u"], hostf["v"], hostf["w"] if dim == 3 else None,
                                 hostf["T"])
            cav.step(args.inner)
            cav.get_macro_into(pout["rho"], pout["u"], pout["v"], pout["w"] if dim == 3 else None, pout["T"])
        f1.record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        barrier()
        ems = max_over_ranks(f0.elapsed_time(f1))
        h2d = nfield * nn * 8
        d2h = nfield * nn * 8
        e2e = {"value": world * nn * iters / (ems / 1e3) / 1e6, "unit": "MLUPS", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "wall_s": wall,
               "path": "lbm_init_equilibrium (pinned host fields) + lbm_step + lbm_get_macro (pinned)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_sample(wl)

    # the second half of the headline metric, beside the throughput: time to a
    # steady state on the first held-out cavities, both arms timed here
    tts = None
    if rank == 0 and world == 1 and args.steady_cases > 0:
        tts = time_to_steady(pkg, args.steady_cases, args.steady_max_steps, local, args.steady_extrapolate)

    if rank == 0:
        line = {
            "metric": "MLUPS", "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.storage,
            "data": "synthetic", "config": config_of(args, wl), "iterations_per_step": args.inner,
            "kernel_config": kernel_config(cav, pkg),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "bytes_per_lup": bpl,
                         "kernel": ("k_march" if cav.kernel == "march" else "k_step") + ("3d" if dim == 3 else "2d"),
                         "ms_per_launch": ms_launch, "frac_of_8TBps": achieved / 8000.0},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
            "time_to_steady": tts,
        }
        print(json.dumps(line), flush=True)
    cav.close()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
