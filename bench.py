"""Benchmark of the explicit MPM substep on B200 (particle-substeps/s).

Workload: two colliding NEO_HOOKEAN spheres (r = 0.12, +-2 m/s)
on a 128^3 grid, 8 particles per cell (242,664 particles), slip walls,
gravity, dt = 5e-5.  One step = one substep over the whole scene.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Timing: W untimed substeps, then K substeps each timed with CUDA events on the
library's stream, the L2 flushed (a 512 MB write) before every timed substep;
value = particles * K / (sum of substep times), max over ranks.  `e2e` goes
through the public C ABI with host buffers: per step, upload of the scene from
pinned host memory, the scene's full run of substeps (CUDA-graph replay),
download of the particle state.  `--impl reference` times the reference's own
CPU driver (compiled from its sources into oracle/_ref) on the host cores.
Multi-GPU: independent replicas, one per rank (the substep does not shard).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "particle-substeps/s"
WORKLOAD = "spheres3d-128^3-neohookean-8ppc-fp32"
LARGE_WORKLOAD = "dam3d-256^3-corotated-8ppc-fp32"
ALG_BYTES = {"p2g": 112, "g2p": 144, "substep": 256}    # bytes per particle (FP32, 3D)
# plastic state read and written by G2P per particle: snow Fp, mu0, lambda0;
# sand Fp, plastic_def, rho_F, sigma_Y, vc
PLASTIC_BYTES = {1: 88, 2: 104}
IMPLICIT_LEAD = 12                                      # implicit leg: substeps run before timing (contact)
SNOW_LEAD_SUBSTEPS = 600                                # plastic legs: substeps run before timing
GRID_BYTES_PER_NODE = 48                                # grid update: read 16, write 32


def chosen(report):
    """The autotuner's full report goes to stderr; the JSON line keeps the chosen shape."""
    print("autotune: " + report, file=sys.stderr, flush=True)
    return report.split("chosen", 1)[-1].strip() if "chosen" in report else report


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if len(s) >= 9 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) >= 9 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            if len(s) >= 9:
                for nm, v in zip(names, s[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def dist_setup(args):
    from physbam_b200 import replicas
    return replicas.rank_env()


def reference_arm(args):
    """Time the reference's own CPU driver (oracle/_ref, all host threads) on the workload."""
    world, rank, _ = dist_setup(args)
    if rank != 0:
        return 0
    import oracle
    from physbam_b200 import scenes as S
    scene = S.spheres_3d()
    cores = os.cpu_count() or 1
    nsteps = args.warmup + args.steps
    if oracle.ref_available():
        s = scene.copy()
        s.nsteps = nsteps
        _, t = oracle.run_reference(s, [], threads=cores, timing=True)
        secs = t["step_seconds"][args.warmup:]
        kind = "reference"
        sample = "full scene (%d particles), %d timed substeps after %d warm-up, PhysBAM MPM_DRIVER FP64, %d OpenMP threads" % (
            scene.n, args.steps, args.warmup, cores)
    else:
        st = oracle.State(scene)
        oracle.run(st, args.warmup)
        t0 = time.perf_counter()
        oracle.run(st, args.steps)
        secs = [(time.perf_counter() - t0) / args.steps] * args.steps
        kind, cores = "port", 1
        sample = "full scene (%d particles), %d substeps, C restatement FP64, 1 thread" % (scene.n, args.steps)
    total = float(sum(secs))
    value = scene.n * args.steps / total
    line = {"metric": METRIC, "value": value, "unit": METRIC, "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded jittered-in-cell seeding, numpy PCG64 seed 1234)",
            "config": {"workload": WORKLOAD, "particles": scene.n, "grid": "128^3", "dt": scene.dt},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_sample(scene, seconds_budget=20.0):
    """Bounded CPU sample of the same workload (rank 0, N=1 only)."""
    import oracle
    cores = os.cpu_count() or 1
    if oracle.ref_available():
        s = scene.copy()
        s.nsteps = 12
        _, t = oracle.run_reference(s, [], threads=cores, timing=True)
        secs = t["step_seconds"][2:]
        return {"value": scene.n * len(secs) / sum(secs), "unit": METRIC, "cores": cores, "kind": "reference",
                "sample": "full scene (%d particles), 10 substeps after 2 warm-up, PhysBAM MPM_DRIVER FP64, %d OpenMP threads"
                          % (scene.n, cores)}
    st = oracle.State(scene)
    t0 = time.perf_counter()
    oracle.run(st, 2)
    dt = (time.perf_counter() - t0) / 2
    return {"value": scene.n / dt, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": "full scene (%d particles), 2 substeps, C restatement FP64, 1 thread" % scene.n}


def kernels_per_substep(scene, p2g_variant=0):
    """Our kernels launched per fast-path substep: the block scan (k_bins), the
    routing of the slots (k_route), P2G, the grid update and G2P."""
    return 5


def read_traffic(kernel, workload=WORKLOAD):
    """Per-launch DRAM traffic of `kernel` on `workload` from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 3 and parts[0] == kernel and parts[1] == workload:
                return float(parts[2])
    return None


def hold_gpu(ms=1.0):
    """A bounded spin kernel on the current stream: the host queues the next
    substep's launches and events while it runs, so that the per-kernel event
    times measure the kernels back to back rather than the host's launch gaps."""
    import torch
    torch.cuda._sleep(int(ms * 2e6))


def measure_substeps(drv, stream, flush, steps, warmup, dist=None, clock_index=None):
    """Warm up, take per-kernel shares from an eager event-timed pass, then time
    `steps` graph-replayed substeps, each bracketed by CUDA events on the
    library's stream with the L2 flushed before it.  Returns (ms_total, kernel
    times, clock summary)."""
    import torch
    drv.advance(max(warmup, 3))
    drv.synchronize()
    drv.set_timing(True)
    for _ in range(4):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
            hold_gpu()
        drv.Advance_One_Time_Step()
    drv.synchronize()
    ktimes = drv.get_timing()
    drv.set_timing(False)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(clock_index) if clock_index is not None else None
    if clk:
        clk.__enter__()
    for k in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
            evs[k][0].record(stream)
        drv.advance(1)
        with torch.cuda.stream(stream):
            evs[k][1].record(stream)
    torch.cuda.synchronize()
    if clk:
        clk.__exit__(None, None, None)
    drv.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in evs)
    return ms, ktimes, (clk.summary() if clk else None)


def roofline_of(ktimes, n, peak, peak_kind, workload):
    shares = {k: v[0] for k, v in ktimes.items()}
    top = max(shares, key=shares.get)
    per_launch_ms = ktimes[top][0] / max(ktimes[top][1], 1)
    alg = {"fast_p2g": ALG_BYTES["p2g"] * n, "fast_g2p": ALG_BYTES["g2p"] * n}.get(top)
    if not alg:
        return {"bound": "hbm", "kernel": top, "achieved": None, "peak": peak, "unit": "GB/s", "frac": None,
                "traffic": None, "note": "dominant kernel has no algorithmic byte count"}
    achieved = alg / (per_launch_ms / 1e3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_kind": peak_kind, "kernel": top, "traffic": read_traffic(top, workload),
            "alg_bytes_per_launch": alg, "ms_per_launch": per_launch_ms}


def our_arm(args):
    import torch
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    from physbam_b200 import replicas
    dist = replicas.init("nccl", timeout_s=120)
    from physbam_b200 import driver as D
    from physbam_b200 import scenes as S

    peak, peak_kind = measured_peaks()
    if args.scene:
        return profile_case(args, D, S)
    scene = S.spheres_3d()
    n = scene.n
    drv = D.MPM_DRIVER(scene, precision=D.FP32, path=D.PATH_FAST)
    stream = torch.cuda.Stream()
    drv.set_stream(stream.cuda_stream)
    drv.set_scene_particles(scene)
    tuned = chosen(drv.autotune(substeps=5, cold_l2=True))   # the timed substeps below run with the L2 flushed
    shape = drv.get_launch_shape()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    ms, ktimes, clocks = measure_substeps(drv, stream, flush, args.steps, args.warmup, dist, local)
    ms_max = replicas.max_over_ranks(ms, dist, "cuda")
    if dist:
        dist.barrier()
    value = world * n * args.steps / (ms_max / 1e3)
    drv.close()

    # e2e through the public API with pinned host buffers
    d = 3
    # page-locked buffers in the C-ABI layout (F, B column-major per particle,
    # as PhysBAM's MATRIX stores them), filled once outside the timed region
    pin = lambda shape, dt=torch.float32: torch.empty(shape, dtype=dt, pin_memory=True).numpy()
    hX, hV, hF, hB = pin((n, d)), pin((n, d)), pin((n, d * d)), pin((n, d * d))
    hm, hvol, hmu, hla = pin(n), pin(n), pin(n), pin(n)
    hX[:], hV[:] = scene.X, scene.V
    hF[:], hB[:] = np.swapaxes(scene.F, 1, 2).reshape(n, 9), np.swapaxes(scene.B, 1, 2).reshape(n, 9)
    hm[:], hvol[:], hmu[:], hla[:] = scene.mass, scene.volume, scene.mu, scene.lam
    oX, oV, oF, oB, ovalid = pin((n, d)), pin((n, d)), pin((n, d * d)), pin((n, d * d)), pin(n, torch.uint8)
    e2e_steps = max(1, min(args.steps, 3))
    frame = scene.nsteps
    h2d = n * 4 * (3 + 3 + 9 + 9 + 4)
    d2h = n * (4 * (3 + 3 + 9 + 9) + 1)
    e2e_drv = D.MPM_DRIVER(scene, precision=D.FP32, path=D.PATH_FAST)
    e2e_drv.set_launch_shape(*shape)   # the autotuner's choice above (mpm_set_launch_shape)
    e2e_drv.set_particles_native(hX, hV, hF, hB, hm, hvol, hmu, hla)
    e2e_drv.advance(2)
    e2e_drv.get_particles_native(oX, oV, oF, oB, ovalid)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_drv.set_particles_native(hX, hV, hF, hB, hm, hvol, hmu, hla)
        e2e_drv.advance(frame)
        e2e_drv.get_particles_native(oX, oV, oF, oB, ovalid)
    e2e_s = time.perf_counter() - t0
    e2e_value = world * n * frame * e2e_steps / replicas.max_over_ranks(e2e_s, dist, "cuda")
    e2e_drv.close()
    assert ovalid.sum() > 0

    substep_ms = ms_max / args.steps
    roof = roofline_of(ktimes, n, peak, peak_kind, WORKLOAD)
    total_k = sum(v[0] for v in ktimes.values())

    large = batch = adjoint = plain = snow = sand = implicit = extras = None
    if world == 1 and not args.no_plain:
        plain = measure_plain_fp64(args, D, S, stream, flush, substep_ms)
    if world == 1 and not args.no_snow:
        snow = measure_plastic(args, D, S, stream, flush, peak, substep_ms, S.snowballs_3d(),
                               "snowballs3d-128^3-corotated-8ppc-clamp-fp32")
        sand = measure_plastic(args, D, S, stream, flush, peak, substep_ms, S.sand_3d(),
                               "sand3d-128^3-hencky-8ppc-druckerprager-fp32")
    if world == 1 and not args.no_implicit:
        implicit = measure_implicit(args, D, S, stream, flush)
    if world == 1 and not args.no_extras:
        extras = measure_collision_extras(args, D, S, stream, flush, substep_ms)
    if world == 1 and not args.no_large:
        large = measure_large(args, D, S, stream, flush, peak, peak_kind)
    if not args.no_batch:
        batch = measure_batch(args, D, S, stream, flush, peak, dist)
    if world == 1 and not args.no_adjoint:
        adjoint = measure_adjoint(D, S, stream)
    par = None
    if rank == 0 and world == 1 and not args.no_parity:
        par = measure_parity(args)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline_sample(scene)
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": substep_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            # the precision and adjoint targets, short and early in the line
            "fp32_over_plain_fp64": plain["fast_fp32_speedup"] if plain else None,
            "cfg2_pos_rel_err": par["spheres3d-128"]["X"] if par and "spheres3d-128" in par else None,
            "cfg2_pos_rel_err_vs_plain_fp64": plain["pos_rel_err_vs_fast_fp32"] if plain else None,
            "bwd_over_fwd_plain": adjoint["bwd_over_fwd_plain"] if adjoint else None,
            "bwd_over_fwd_fast": adjoint["bwd_over_fwd_fast"] if adjoint else None,
            "parity": par,
            "data": "synthetic (seeded jittered-in-cell seeding, numpy PCG64 seed 1234)",
            "config": {"workload": WORKLOAD, "particles": n, "grid": "128^3", "dt": scene.dt,
                       "l2": "flushed before every timed substep (512 MB write)",
                       "parallelism": "replicas" if world > 1 else "single"},
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "step": "mpm_set_particles + %d substeps (mpm_advance, CUDA graph) + mpm_get_particles, "
                            "pinned host buffers in the C-ABI layout" % frame},
            "gpu_launches": kernels_per_substep(scene, shape[0]) * args.steps,
            "autotune": tuned,
            "roofline": roof,
            "substep_roofline": {"achieved": ALG_BYTES["substep"] * n / (substep_ms / 1e3) / 1e9, "peak": peak,
                                 "unit": "GB/s", "frac": ALG_BYTES["substep"] * n / (substep_ms / 1e3) / 1e9 / peak,
                                 "alg_bytes_per_particle": ALG_BYTES["substep"]},
            "kernel_ms_per_substep": {k: v[0] / max(v[1], 1) for k, v in ktimes.items()},
            "kernel_share": {k: v[0] / total_k for k, v in ktimes.items()},
            "plain_fp64": plain,
            "implicit": implicit,
            "snow": snow,
            "sand": sand,
            "collision_extras": extras,
            "large_config": large,
            "batch_config": batch,
            "adjoint": adjoint,
            "cpu_baseline": cpu,
            "clocks": clocks}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def measure_batch(args, D, S, stream, flush, peak, dist=None):
    """256 independent scenes (grid side from {32,48,64,96}, boxes of seeded size,
    4-8 ppc, both models) in one handle; launch shapes from the autotuner.  With
    N ranks the scenes are split into N partitions of similar particle totals
    (no collective on the data path); the whole job's rate is all particles over
    the slowest rank's time."""
    from physbam_b200 import replicas
    world, rank, _ = replicas.rank_env()
    every = S.batch_scenes(seed=1234, count=256)
    mine = replicas.partition_scenes([s.n for s in every], world)[rank]
    scenes = [every[i] for i in mine]
    n_all = sum(s.n for s in every)
    drv = D.MPM_BATCH(scenes)
    drv.set_stream(stream.cuda_stream)
    drv.set_scene_particles(dtype=np.float32)
    report = chosen(drv.autotune(substeps=3, cold_l2=True))
    steps = max(5, min(args.steps, 20))
    ms, ktimes, _ = measure_substeps(drv, stream, flush, steps, 3, dist)
    drv.close()
    ms = replicas.max_over_ranks(ms, dist, "cuda")
    sub = ms / steps
    n = n_all
    # the substep is 5 kernels replayed from a graph: what one persistent launch
    # could save at most is the time between them
    kernel_sum = sum(v[0] / max(v[1], 1) for v in ktimes.values())
    return {"workload": "batch256-3d-grids{32,48,64,96}-fp32", "scenes": len(every), "particles": n,
            "partition": "%d ranks, %d scenes on rank 0" % (world, len(mine)) if world > 1 else "single",
            "scaling": "strong",
            "steps": steps, "ms_per_step": sub, "value": n * steps / (ms / 1e3), "unit": METRIC,
            "substep_roofline": {"achieved": ALG_BYTES["substep"] * n / (sub / 1e3) / 1e9, "peak": peak,
                                 "unit": "GB/s", "frac": ALG_BYTES["substep"] * n / (sub / 1e3) / 1e9 / peak},
            "autotune": report,
            "kernel_ms_per_substep": {k: v[0] / max(v[1], 1) for k, v in ktimes.items()},
            "launch_gaps_ms_per_step": sub - kernel_sum}


def measure_plain_fp64(args, D, S, stream, flush, fast_ms):
    """The same workload on the plain FP64 path (reference layout, one thread per
    particle, global atomics): the FP32 fast path's speed-up over it."""
    scene = S.spheres_3d()
    drv = D.MPM_DRIVER(scene, precision=D.FP64, path=D.PATH_PLAIN)
    drv.set_stream(stream.cuda_stream)
    drv.set_scene_particles(scene)
    steps = max(5, min(args.steps, 20))
    ms, ktimes, _ = measure_substeps(drv, stream, flush, steps, 3)
    drv.close()
    sub = ms / steps
    # precision beside the speed-up: both paths over the scene's 200 substeps
    finals = []
    for prec, path in ((D.FP64, D.PATH_PLAIN), (D.FP32, D.PATH_FAST)):
        d = D.MPM_DRIVER(scene, precision=prec, path=path)
        d.set_stream(stream.cuda_stream)
        d.set_scene_particles(scene)
        d.advance(scene.nsteps)
        finals.append(d.get_particles()["X"])
        d.close()
    err = float(np.linalg.norm(finals[1] - finals[0]) / np.linalg.norm(finals[0]))
    return {"workload": WORKLOAD.replace("fp32", "fp64-plain"), "steps": steps, "ms_per_step": sub,
            "value": scene.n * steps / (ms / 1e3), "unit": METRIC, "fast_fp32_speedup": sub / fast_ms,
            "pos_rel_err_vs_fast_fp32": err,
            "kernel_ms_per_substep": {k: v[0] / max(v[1], 1) for k, v in ktimes.items()}}


def measure_plastic(args, D, S, stream, flush, peak, elastic_ms, scene, workload):
    """Two balls with the geometry of the headline case (128^3, 8 ppc) and
    plasticity after every G2P, fused into the fast path's G2P: snow
    (COROTATED_FIXED + MPM_PLASTICITY_CLAMP, Stomakhin et al. 2013 parameters)
    or sand (St. Venant-Kirchhoff Hencky + MPM_DRUCKER_PRAGER, Mast et al.
    hardening).  The cost of plasticity against the elastic headline."""
    n = scene.n
    drv = D.MPM_DRIVER(scene, precision=D.FP32, path=D.PATH_FAST)
    drv.set_stream(stream.cuda_stream)
    drv.set_scene_particles(scene)
    # timed mid-collision: the balls touch after ~300 substeps, and from then on
    # the clamp acts and hardens (before, the SVD is skipped for every particle)
    drv.advance(SNOW_LEAD_SUBSTEPS)
    tuned = chosen(drv.autotune(substeps=3, cold_l2=True))
    steps = max(5, min(args.steps, 20))
    ms, ktimes, _ = measure_substeps(drv, stream, flush, steps, 3)
    plastic = drv.get_plastic_state(np.float32)
    drv.close()
    sub = ms / steps
    g2p = ktimes.get("fast_g2p")
    g2p_ms = g2p[0] / max(g2p[1], 1) if g2p else None
    extra = PLASTIC_BYTES[scene.plasticity.kind]
    g2p_bytes = (ALG_BYTES["g2p"] + extra) * n
    if scene.plasticity.kind == S.PLASTICITY_CLAMP:
        frac = float(np.mean(np.abs(plastic["mu"] / plastic["mu0"] - 1.0) > 1e-4))
    else:
        frac = float(np.mean(plastic["pdef"] > 0))
    return {"workload": workload, "particles": n, "steps": steps,
            "timed_after_substeps": SNOW_LEAD_SUBSTEPS,
            "ms_per_step": sub, "value": n * steps / (ms / 1e3), "unit": METRIC,
            "over_elastic_headline": sub / elastic_ms,
            "plastic_fraction": frac,
            "g2p_roofline": None if g2p_ms is None else {
                "achieved": g2p_bytes / (g2p_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                "frac": g2p_bytes / (g2p_ms / 1e3) / 1e9 / peak,
                "alg_bytes_per_particle": ALG_BYTES["g2p"] + extra},
            "autotune": tuned,
            "kernel_ms_per_substep": {k: v[0] / max(v[1], 1) for k, v in ktimes.items()}}


def measure_collision_extras(args, D, S, stream, flush, elastic_ms):
    """The headline scene on the fast path with (a) penalty collision objects: a
    penalty slab under the balls and a penalty ball between them, so the
    impulse pre-pass runs for every particle each substep; (b) moving collision
    objects: a sticky paddle turning between the balls and a slip plate sliding
    over them, whose frames the host evaluates and uploads every substep (timed
    one substep per call, each runs eagerly; mpm_advance over several substeps
    would replay a graph).  Their cost against the elastic headline."""
    out = {}
    steps = max(5, min(args.steps, 20))
    pen = S.spheres_3d()
    pen.penalty = S.Penalty([S.CollisionObject(S.BOX, S.SLIP, 0.0, [-1, -1, -1], [2, 0.39, 2]),
                             S.CollisionObject(S.SPHERE, S.SLIP, 0.0, [0.5, 0.5, 0.5], [0.05, 0, 0])])
    mov = S.spheres_3d()
    mov.objects = mov.objects + [
        S.CollisionObject(S.BOX, S.STICK, 0.0, [-0.01, -0.15, -0.15], [0.01, 0.15, 0.15],
                          motion=S.Motion([0.5, 0.5, 0.5], [0.0, 0.0, 0.0], [0.0, 3.0, 0.0])),
        S.CollisionObject(S.BOX, S.SLIP, 0.3, [-0.2, -0.01, -0.2], [0.2, 0.01, 0.2],
                          motion=S.Motion([0.5, 0.63, 0.5], [0.5, -1.0, 0.0], [0.0, 0.0, 0.0]))]
    for key, scene, workload in (("penalty", pen, "spheres3d-128^3-neohookean-8ppc-fp32 + 2 penalty objects"),
                                 ("moving", mov, "spheres3d-128^3-neohookean-8ppc-fp32 + 2 moving objects")):
        drv = D.MPM_DRIVER(scene, precision=D.FP32, path=D.PATH_FAST)
        drv.set_stream(stream.cuda_stream)
        drv.set_scene_particles(scene)
        chosen(drv.autotune(substeps=3, cold_l2=True))
        ms, ktimes, _ = measure_substeps(drv, stream, flush, steps, 3)
        drv.close()
        sub = ms / steps
        out[key] = {"workload": workload, "particles": scene.n, "steps": steps, "ms_per_step": sub,
                    "value": scene.n * steps / (ms / 1e3), "unit": METRIC, "over_elastic_headline": sub / elastic_ms,
                    "kernel_ms_per_substep": {k: v[0] / max(v[1], 1) for k, v in ktimes.items()}}
    return out


def measure_implicit(args, D, S, stream, flush):
    """The headline geometry with the reference's default solve: backward Euler
    (Newton + CG + Wolfe line search, MPM_EXAMPLE's default tolerances) at a
    40x larger step, dt = 2e-3, timed once the spheres are in contact (after
    IMPLICIT_LEAD substeps), on the plain path in FP64 and FP32; beside it the
    reference's own implicit driver on the host cores, same scene, same steps."""
    import torch
    import oracle
    scene = S.spheres_3d(dt=2e-3)
    scene.implicit = S.Implicit()
    out = {"workload": "spheres3d-128^3-neohookean-8ppc-implicit-dt2e-3", "particles": scene.n, "dt": scene.dt,
           "timed_after_substeps": IMPLICIT_LEAD}
    steps = max(3, min(args.steps, 8))
    for name, prec in (("fp64", D.FP64), ("fp32", D.FP32)):
        drv = D.MPM_DRIVER(scene, precision=prec, path=D.PATH_PLAIN)
        drv.set_stream(stream.cuda_stream)
        drv.set_scene_particles(scene)
        for _ in range(IMPLICIT_LEAD):
            drv.Advance_One_Time_Step()
        drv.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        newton = cg = 0
        for k in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(k))
                evs[k][0].record(stream)
            drv.Advance_One_Time_Step()
            with torch.cuda.stream(stream):
                evs[k][1].record(stream)
            st = drv.implicit_stats()
            newton += st["newton_iterations"]
            cg += st["krylov_iterations"]
        torch.cuda.synchronize()
        drv.close()
        ms = sum(a.elapsed_time(b) for a, b in evs) / steps
        out[name] = {"ms_per_step": ms, "value": scene.n / (ms / 1e3), "unit": METRIC,
                     "newton_per_step": newton / steps, "cg_per_step": cg / steps}
    if oracle.ref_available() and not args.no_cpu:
        s = scene.copy()
        s.nsteps = IMPLICIT_LEAD + 3
        cores = os.cpu_count() or 1
        _, t = oracle.run_reference(s, [], threads=cores, timing=True)
        secs = t["step_seconds"][IMPLICIT_LEAD:]
        ref_ms = 1e3 * sum(secs) / len(secs)
        out["reference"] = {"ms_per_step": ref_ms, "value": scene.n / (ref_ms / 1e3), "unit": METRIC, "cores": cores,
                            "kind": "reference",
                            "sample": "3 substeps after the same %d lead substeps, PhysBAM MPM_DRIVER implicit FP64, "
                                      "%d OpenMP threads" % (IMPLICIT_LEAD, cores)}
        out["fp64_speedup_over_reference"] = ref_ms / out["fp64"]["ms_per_step"]
    return out


def measure_adjoint(D, S, stream):
    """The differentiable cube: 64^3, 64 substeps, checkpoint every 8.  The FP32
    rollout with checkpoints (mpm_diff_forward, plain path) and its adjoint
    (mpm_diff_backward) through the C ABI on device arrays, beside the fast FP32
    forward of the same 64 substeps (mpm_advance); each timed with CUDA events on
    the library's stream, best of 3 after one warm-up.  Twice: with the default
    tape budget (the forward keeps every substep, the backward recomputes
    nothing) and with checkpoints only (each segment recomputed)."""
    import torch
    scene = S.cube_3d()
    n = scene.n
    drv = D.MPM_DRIVER(scene, precision=D.FP32, path=D.PATH_PLAIN)
    drv.set_stream(stream.cuda_stream)
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")
    X, V = t(scene.X), t(scene.V)
    Fc = t(np.swapaxes(scene.F, 1, 2).reshape(n, 9))
    Bc = t(np.swapaxes(scene.B, 1, 2).reshape(n, 9))
    m, vol, mu, lam = t(scene.mass), t(scene.volume), t(scene.mu), t(scene.lam)
    g = [torch.ones_like(X) * 1e-3, torch.zeros_like(V), torch.zeros_like(Fc), torch.zeros_like(Bc)]

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b)

    fwd, bwd, fwd_ck, bwd_ck, fast = [], [], [], [], []
    for budget, fl, bl in ((-1, fwd, bwd), (0, fwd_ck, bwd_ck)):   # every substep kept; checkpoints only
        drv.set_diff_tape_budget(budget)
        for it in range(4):
            drv.set_particles_device(X, V, Fc, Bc, m, vol, mu, lam)
            f = timed(lambda: drv.diff_forward(64, 8))
            b = timed(lambda: drv.diff_backward(*g))
            if it:
                fl.append(f)
                bl.append(b)
    drv.close()
    fd = D.MPM_DRIVER(scene, precision=D.FP32, path=D.PATH_FAST)
    fd.set_stream(stream.cuda_stream)
    for it in range(4):
        fd.set_scene_particles(scene)
        torch.cuda.synchronize()
        ms = timed(lambda: fd.advance(64))
        if it:
            fast.append(ms)
    fd.close()
    f, b, ff, fc, bc = min(fwd), min(bwd), min(fast), min(fwd_ck), min(bwd_ck)
    return {"workload": "cube3d-64^3-corotated-8ppc, 64 substeps, checkpoint every 8, fp32", "particles": n,
            "fwd_plain_ms": f, "bwd_ms": b, "fwd_fast_ms": ff, "bwd_over_fwd_plain": b / f,
            "bwd_over_fwd_fast": b / ff,
            "checkpoints_only": {"fwd_plain_ms": fc, "bwd_ms": bc, "bwd_over_fwd_plain": bc / fc,
                                 "bwd_over_fwd_fast": bc / ff,
                                 "note": "mpm_set_diff_tape_budget(0): the backward recomputes each segment"},
            "timing": "CUDA events on the library's stream around each C-ABI call, best of 3 after a warm-up"}


def measure_parity(args):
    """Per-quantity relative L2 error of the FP32 fast path against the reference's
    own FP64 build (oracle/_ref, all host threads) after the last substep: the two
    spheres (200 substeps), the 64^3 dam break (100), the cube (64) and eleven
    scenes of the 256-scene batch run in one batch handle.  Outside every timed
    region; the checker, not a measurement of speed."""
    import oracle
    from oracle import parity
    if not oracle.ref_available():
        return None
    table = {}
    for name in sorted(parity.SINGLE):
        table[name] = parity.single_table(name)
    table.update(parity.batch_table())
    return parity.compact(table)


def profile_case(args, D, S):
    """Small single-scene run for profilers: `--scene NAME --grid G` (no e2e, no CPU, no flush).
    Prints one JSON line with the per-kernel times; used to make the ncu summaries."""
    import torch
    def spheres_implicit(**kw):
        s = S.spheres_3d(dt=2e-3, **kw)
        s.implicit = S.Implicit()
        return s
    make = {"spheres3d": S.spheres_3d, "dam3d": S.dam_3d, "cube3d": S.cube_3d,
            "snowballs3d": S.snowballs_3d, "sand3d": S.sand_3d, "spheres3d_implicit": spheres_implicit}[args.scene]
    scene = make(G=args.grid) if args.grid else make()
    if scene.implicit is not None:     # the plain path, FP64, from the contact phase on
        drv = D.MPM_DRIVER(scene, precision=D.FP64, path=D.PATH_PLAIN)
        drv.set_scene_particles(scene)
        for _ in range(IMPLICIT_LEAD + args.warmup):
            drv.Advance_One_Time_Step()
        drv.synchronize()
        drv.set_timing(True)
        for _ in range(args.steps):
            drv.Advance_One_Time_Step()
        drv.synchronize()
        kt = drv.get_timing()
        drv.close()
        print(json.dumps({"scene": args.scene, "particles": scene.n, "steps": args.steps,
                          "kernel_ms_per_substep": {k: v[0] / max(args.steps, 1) for k, v in kt.items()}}), flush=True)
        return 0
    drv = D.MPM_DRIVER(scene, precision=D.FP32, path=D.PATH_FAST)
    stream = torch.cuda.Stream()
    drv.set_stream(stream.cuda_stream)
    if args.shape:
        drv.set_launch_shape(*[int(x) for x in args.shape.split(",")])
    drv.set_scene_particles(scene, dtype=np.float32)
    if scene.plasticity is not None:
        drv.advance(SNOW_LEAD_SUBSTEPS)   # into the collision, where the clamp acts
    drv.advance(args.warmup)
    drv.synchronize()
    drv.set_timing(True)
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            hold_gpu()
        drv.Advance_One_Time_Step()
    drv.synchronize()
    kt = drv.get_timing()
    drv.close()
    print(json.dumps({"scene": args.scene, "grid": args.grid, "particles": scene.n, "steps": args.steps,
                      "kernel_ms_per_substep": {k: v[0] / max(v[1], 1) for k, v in kt.items()}}), flush=True)
    return 0


def measure_large(args, D, S, stream, flush, peak, peak_kind):
    """The 256^3 dam-break scene (36M particles): the HBM-bound regime of the same kernels."""
    scene = S.dam_3d()
    n = scene.n
    drv = D.MPM_DRIVER(scene, precision=D.FP32, path=D.PATH_FAST)
    drv.set_stream(stream.cuda_stream)
    drv.set_scene_particles(scene, dtype=np.float32)
    del scene.F, scene.B
    tuned = chosen(drv.autotune(substeps=2, cold_l2=True))
    steps = max(5, min(args.steps, 20))
    ms, ktimes, _ = measure_substeps(drv, stream, flush, steps, 3)
    drv.close()
    sub = ms / steps
    total_k = sum(v[0] for v in ktimes.values())
    return {"workload": LARGE_WORKLOAD, "particles": n, "steps": steps, "ms_per_step": sub,
            "value": n * steps / (ms / 1e3), "unit": METRIC,
            "substep_roofline": {"achieved": ALG_BYTES["substep"] * n / (sub / 1e3) / 1e9, "peak": peak,
                                 "unit": "GB/s", "frac": ALG_BYTES["substep"] * n / (sub / 1e3) / 1e9 / peak},
            "roofline": roofline_of(ktimes, n, peak, peak_kind, LARGE_WORKLOAD),
            "autotune": tuned,
            "kernel_ms_per_substep": {k: v[0] / max(v[1], 1) for k, v in ktimes.items()},
            "kernel_share": {k: v[0] / total_k for k, v in ktimes.items()}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-large", action="store_true", help="skip the 256^3 dam-break measurement")
    ap.add_argument("--no-batch", action="store_true", help="skip the 256-scene batched measurement")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the forward/backward timing")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 path on the same workload")
    ap.add_argument("--no-implicit", action="store_true", help="skip the backward-Euler measurement")
    ap.add_argument("--no-snow", action="store_true", help="skip the snow and sand (plasticity) measurements")
    ap.add_argument("--no-extras", action="store_true", help="skip the penalty and moving-object measurements")
    ap.add_argument("--no-parity", action="store_true", help="skip the FP32-vs-reference-FP64 error table")
    ap.add_argument("--scene", choices=["spheres3d", "dam3d", "cube3d", "snowballs3d", "sand3d", "spheres3d_implicit"],
                    help="profiling run of one scene only")
    ap.add_argument("--grid", type=int, default=0, help="grid cells per side for --scene")
    ap.add_argument("--shape", default="", help="launch shape for --scene: P2G variant,G2P threads,CTA multiplier")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)
    return our_arm(args)


if __name__ == "__main__":
    sys.exit(main())
