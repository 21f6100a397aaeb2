"""Throughput of the ssol_solve realisation loop on B200.

Workload (default): the 1000-heliostat radial-staggered field with a 64x64
per-primitive receiver (workloads.heliostat_field), 1e8 realisations per
step, FP32 geometry/BSDFs and FP64 tallies.

value: Mpaths/s with the scene resident in HBM (a plan created once; each
       step is one launch of `paths` realisations on the current CUDA
       stream), CUDA-event timed over the K steps, L2 flushed between steps.
e2e:   the same metric through the public C API, `ssol_solve` per step:
       host snapshot, BVH build, host->device copy, launch, device->host
       tally read and estimator construction, wall-clock timed around the
       synchronous call.
--impl reference: the CPU restatement of the reference solver (oracle/)
       on all host cores, each step a bounded sample of the same workload.
Multi-GPU (torchrun): each rank traces a disjoint range of realisations of
the same scene (weak scaling, no collective on the data path); the time is
the max over ranks. After the timed region the ranks' tally vectors are
all-reduced in place over NCCL (the one collective), so that the line's
estimate is that of all ranks' realisations.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "solstice-solver_b200")
sys.path.insert(0, PKG)
ORACLE_LIB = os.path.join(ROOT, "oracle", "_build", "liboracle_ssol.so")
METRIC = "Mpaths/s"
WORKLOAD = ("1000 flat 10x10 heliostats (radial staggered, r 100-600 m, Beckmann "
            "2 mrad, reflectivity 0.9), 12x12 receiver at 100 m with 64x64 per-primitive "
            "map, pillbox sun 4.65 mrad el 30 az 180 DNI 900, extinction 1e-4/m")


# DRAM bytes per path of the realisation kernel, from ncu captures of launches
# of the same scenes, the variants without work counters (field: one sorted
# chunk of 2^24 paths at 3 blocks per SM; beam-down: 4e6 paths)
# (dram__bytes_read.sum + dram__bytes_write.sum);
# the traffic scales with the paths traced (per-thread frames written back)
DRAM_BYTES_PER_PATH = {"field": (2202.1e6 + 15599.4e6) / 16777216,
                       "beamdown": (892.0e6 + 3562.1e6) / 4e6}  # beam-down: id order

# Kernels of one plain launch of n realisations: below 6e6 the realisation
# kernel alone; from 6e6 on, per chunk of at most 2^24 realisations, the
# coherent order's presort (count, scan, scatter) and the realisation kernel
# (every bench scene samples more than one and fewer than 12288 primitives)
SORT_MIN, SORT_CHUNK = 6_000_000, 1 << 24


def launches_per_plain_launch(n):
    return 1 if n < SORT_MIN else 4 * ((n + SORT_CHUNK - 1) // SORT_CHUNK)
# Both passes of the adjoint kernel on the field, from a capture of 4e6 paths
ADJOINT_DRAM_BYTES_PER_PATH = (2.76e6 + 26.97e6 + 5.95e6 + 52.99e6) / 4e6
# Same for the batched kernel, from a capture of 32 suns (32245124 paths)
BATCH_DRAM_BYTES_PER_PATH = (4571.5e6 + 19782.1e6) / 32245124


def flops_per_run(st):
    """Algorithmic FP32 work model: 20 FLOP per child slab test (2 per node),
    55 per triangle test, 90 per quadric test, 150 per shaded bounce, 120 per
    primary sample."""
    return (20 * 2 * st["node_visits"] + 55 * st["triangle_tests"]
            + 90 * st["quadric_tests"] + 150 * st["bounces"] + 120 * st["paths"])


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons while running."""
    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        """Start sampling; returns once the first sample is in, so that the
        timed region that follows is covered from its start."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
            return
        t0 = time.time()
        while not self.lines and time.time() - t0 < 3.0 and self.proc.poll() is None:
            time.sleep(0.01)
        self.mark = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        # A region shorter than the sampling period may hold no sample: then
        # the samples just before and just after it bracket it
        mark = getattr(self, "mark", 0)
        t0 = time.time()
        while len(self.lines) <= mark and time.time() - t0 < 0.5 and self.proc.poll() is None:
            time.sleep(0.01)
        self.lines = self.lines[max(0, mark - 1):]
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax = max(smax, float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() in ("active", "0x1", "yes"):
                    reasons.add(n)
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except Exception:
        pass
    return None


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def shard_first(step, rank, world, n):
    """First realisation (relative to the RNG position) of `rank`'s share of
    step `step`: every step hands each rank a disjoint range of n
    realisation ids, so the ranks together trace exactly the ids a single
    GPU would trace in world x more steps."""
    return (step * world + rank) * n


def shard_suns(suns, rank, world):
    """Sun slots of `rank` in the batched form: every world-th sun."""
    return suns[rank::world]


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


BEAMDOWN = ("beam-down tower: 5000 punched 8x8 paraboloid heliostats (surround field, "
            "r <= 440 m, focal = slant range to the secondary), hyperboloid secondary at "
            "120 m (40x40 m, reflectivity 0.95, pillbox microfacet 1.5 mrad), 6x6 ground "
            "receiver (absorptivity 0.9, 30x30 per-primitive map) under a thin-dielectric "
            "window (n 1.5, 20/m, 5 mm), Gaussian sun 2.5 mrad el 60 az 180 DNI 1000")


def build_workload(lib, args):
    import workloads as W
    if args.config == "mirror":
        s, h = W.single_mirror(lib)
        desc = "single 10x10 mirror, 4x4 receiver at 50 m, pillbox 4.65 mrad, DNI 1000"
    elif args.config == "beamdown":
        s, h = W.beam_down(lib)
        desc = BEAMDOWN
    else:
        s, h = W.heliostat_field(lib, n_helio=args.heliostats)
        desc = WORKLOAD if args.heliostats == 1000 else WORKLOAD.replace(
            "1000", str(args.heliostats), 1)
    return s, h, desc


def cpu_reference_rate(args, seconds):
    """Oracle paths/s on all host cores for a sample of about `seconds`."""
    import pyssol as P
    lib = P.Lib(ORACLE_LIB)
    s, h, _ = build_workload(lib, args)
    probe = 20000
    t = time.perf_counter()
    s.solve(probe, seed=123)
    rate = probe / (time.perf_counter() - t)
    # Solves of about a quarter of the sample each, until the sample has run
    # for `seconds` (the probe's rate is only a first guess)
    total_n, dt, k = 0, 0.0, 0
    while dt < seconds and k < 64:
        n = int(min(max(rate * seconds / 4, probe), 5e8))
        t = time.perf_counter()
        est = s.solve(n, seed=124 + k)
        step = time.perf_counter() - t
        del est
        total_n += n
        dt += step
        rate = n / step
        k += 1
    return total_n / dt, total_n, dt


def run_reference(args):
    """CPU restatement of the reference solver on the host cores."""
    rank, world, _ = dist_env()
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("gloo")
        if rank != 0:
            dist.barrier()
            dist.destroy_process_group()
            return
    import pyssol as P
    if not os.path.exists(ORACLE_LIB):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True,
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    lib = P.Lib(ORACLE_LIB)
    s, h, desc = build_workload(lib, args)
    probe = 20000
    t = time.perf_counter()
    s.solve(probe, seed=1)
    rate = probe / (time.perf_counter() - t)
    n = int(min(max(rate * args.ref_step_seconds, probe), args.paths))
    for w in range(args.warmup):
        s.solve(n, seed=100 + w)
    t = time.perf_counter()
    for k in range(args.steps):
        est = s.solve(n, seed=1000 + k)
        del est
    dt = time.perf_counter() - t
    value = args.steps * n / dt / 1e6
    cores = os.cpu_count()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "paths_per_step": n, "l2": "n/a (CPU)",
                   "paths_per_step_note": (
                       "a bounded sample of the %d-realisation step: about %.0f s of "
                       "CPU work per step, so that the whole run ends within minutes; "
                       "paths are independent and the per-solve set-up is below 1 %% "
                       "of a step, so paths/s does not depend on the sample size"
                       % (args.paths, args.ref_step_seconds))},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": "port",
                         "cpu_model": cpu_model(),
                         "sample": "%d realisations per step of the same scene" % n},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def run_b200(args):
    import torch
    import pyssol as P
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    lib = P.load_product()
    s, h, desc = build_workload(lib, args)
    opt = P.options(P.FP64 if args.fp64 else P.FP32, block_size=args.block,
                    waves=args.waves, leaf=args.leaf, min_blocks=args.minb,
                    bvh=BVH_CHOICES[args.bvh])
    tuned_ms = None
    if args.autotune:
        opt, tuned_ms = P.autotune(s, args.autotune_paths, opt, seed=args.seed + 77)
    launch_shape = {"block": opt.block_size, "blocks_per_sm_budget": opt.min_blocks_per_sm,
                    "waves": opt.waves, "bvh_leaf": opt.bvh_leaf_size,
                    "bvh_builder": args.bvh, "autotuned": bool(args.autotune)}
    plan = P.C.c_void_p()
    lib.call("ssol_b200_plan_create", s.scn, P.C.byref(opt), P.C.byref(plan))
    rng = s.rng(seed=args.seed)
    # A dedicated stream: its handle is what the library launches on (a NULL
    # handle would select the plan's own stream, outside these events)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = P.C.c_void_p(stream.cuda_stream)
    assert sp.value, "expected a non-default CUDA stream"
    n = args.paths
    flush = torch.empty(max(1, args.flush_mib) * 1024 * 1024 // 4, dtype=torch.float32,
                        device="cuda")

    def step(k):
        first = shard_first(k, rank, world, n)
        lib.call("ssol_b200_plan_launch", plan, rng, first, n, sp)

    for w in range(args.warmup):
        step(w)
        if args.flush_mib:
            flush.zero_()
    lib.call("ssol_b200_plan_reset", plan, sp)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    ev0.record(stream)
    for k in range(args.steps):
        kev[k][0].record(stream)
        step(args.warmup + k)
        kev[k][1].record(stream)
        if args.flush_mib:
            flush.zero_()
    ev1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    kernel_ms = sum(a.elapsed_time(b) for a, b in kev)
    if dist:
        t = torch.tensor([ms, kernel_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, kernel_ms = float(t[0]), float(t[1])
    # The one collective of the multi-GPU path: each rank's tally vectors
    # (disjoint realisation ranges of one scene) all-reduced in place over
    # NCCL, outside the timed region, so that every rank's plan then holds
    # the tallies of all realisations and builds their merged estimator
    merged_n = args.steps * n
    if dist:
        sums, counts = (torch.as_tensor(x, device="cuda") for x in P.plan_tallies(lib, plan))
        dist.all_reduce(sums)
        dist.all_reduce(counts)
        torch.cuda.synchronize()
        merged_n = args.steps * n * world
    est = P.C.c_void_p()
    res = lib.raw("ssol_b200_plan_finish", plan, rng, merged_n, 0, sp, P.C.byref(est))
    e = P.Estimator(s, est, res)
    g = e.globals()
    lib.raw("ssol_b200_plan_ref_put", plan)
    total_paths = args.steps * n * world
    value = total_paths / (ms * 1e-3) / 1e6
    # The work per path for the roofline model: the timed launches leave the
    # work counters out (the library's default), one counted launch of the
    # same plan shape, outside the timed region, gives them
    st = counted_stats(lib, s, opt, n, args.seed + 99, sp)

    # e2e through the public API
    e2e_value, h2d, d2h = None, 0, 0
    if not args.no_e2e:
        e2e_n = n
        for w in range(1):
            e_w = s.solve(e2e_n, rng=rng)
            del e_w
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        e2e_steps = max(1, min(args.steps, 3))
        for k in range(e2e_steps):
            ek = s.solve(e2e_n, rng=rng)
            sk = ek.stats()
            h2d, d2h = sk["scene_bytes"], sk["tally_bytes"]
            del ek
        dt = time.perf_counter() - t0
        if dist:
            t = torch.tensor([dt], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dt = float(t[0])
        e2e_value = e2e_steps * e2e_n * world / dt / 1e6

    # Precision: this build against the all-FP64 build on identical random
    # numbers (same seed and realisation ids), outside the timed region
    prec = None
    if not args.fp64 and not args.no_fp64_check and rank == 0:
        e32 = s.solve(n, seed=args.seed + 11, options=opt)
        o64 = P.options(P.FP64, block_size=opt.block_size, waves=opt.waves,
                        leaf=opt.bvh_leaf_size, min_blocks=opt.min_blocks_per_sm)
        e64 = s.solve(n, seed=args.seed + 11, options=o64)
        rel = {}
        for name, a, b in ([("global." + k, e32.globals()[k], e64.globals()[k])
                            for k in e64.globals()]
                           + [("receiver." + k, e32.receiver(h["receiver"])[k],
                               e64.receiver(h["receiver"])[k])
                              for k in e64.receiver(h["receiver"])]):
            if b[0] != 0:
                rel[name] = (a[0] - b[0]) / b[0]
        prec = {"paths": n, "max_abs_rel_diff": max(abs(v) for v in rel.values()),
                "rel_diff": rel, "what": "FP32 geometry/BSDF build vs all-FP64 build, "
                "same seed and realisation ids, every global and receiver estimate"}
        del e32, e64

    bvh = None
    if rank == 0 and not args.no_bvh_compare and args.config in ("field", "beamdown", "mirror"):
        bvh = bvh_builders(lib, s, opt, n, stream, sp, flush if args.flush_mib else None)

    peaks = measured_peaks()
    nsm = torch.cuda.get_device_properties(local).multi_processor_count
    sm_mhz = peaks.get("sm_max_mhz", 1965.0)
    fp32_peak = nsm * 128 * 2 * sm_mhz * 1e6 / 1e12
    achieved = (flops_per_run(st) / max(1, st["paths"]) * args.steps * n
                / (kernel_ms * 1e-3) / 1e12 if kernel_ms > 0 else 0.0)
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.fp64 else "f32",
        "data": "synthetic (seeded generator, no public scene)",
        "config": {"workload": desc, "paths_per_step": n, "precision":
                   "FP64" if args.fp64 else "FP32 geometry/BSDF, FP64 tallies",
                   "l2": ("flushed: %d MiB write between steps (scene < 2 MB)" % args.flush_mib
                          if args.flush_mib else "not flushed (profiling run)"),
                   "parallelism": "realisation ranges per GPU" if world > 1 else "1 GPU",
                   "launch": launch_shape},
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "timing": "wall clock around synchronous ssol_solve"},
        "gpu_launches": args.steps * launches_per_plain_launch(n),
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak,
                     "unit": "TFLOP/s", "frac": achieved / fp32_peak if fp32_peak else None,
                     "traffic": (DRAM_BYTES_PER_PATH[args.config] * n
                                 if args.config in DRAM_BYTES_PER_PATH else None),
                     "traffic_source": "ncu dram__bytes_read+write of a launch of the "
                                       "realisation kernel, scaled to paths_per_step "
                                       "(bytes per step: its chunks' launches together)",
                     "timing": "CUDA events around each step: the realisation kernel and "
                               "the coherent order's presort (2.3 % of the step)",
                     "peak_source": "SMs x 128 FP32 lanes x 2 x measured max SM clock "
                                    "(MEASURED_PEAKS.json sm_max_mhz)",
                     "work_model": "20/slab x2 per node + 55/triangle + 90/quadric + "
                                   "150/bounce + 120/path (counted on device)",
                     "counters_source": "one counted launch of paths_per_step paths "
                                        "outside the timed region (the timed launches "
                                        "run the kernel variant without work counters)",
                     "counters_per_path": {k: st[k] / max(1, st["paths"]) for k in
                                           ("rays", "node_visits", "triangle_tests",
                                            "quadric_tests", "bounces")},
                     "kernel_ms": kernel_ms},
        "clocks": clk,
        "precision_vs_fp64": prec,
        "bvh_builders": bvh,
        "estimate": {"absorbed_by_receivers_W": g["absorbed_by_receivers"][0],
                     "rel_se": g["absorbed_by_receivers"][2] / max(1e-30,
                                                                  g["absorbed_by_receivers"][0]),
                     "realisations": merged_n,
                     "what": ("merged over the ranks: plan tallies all-reduced over NCCL"
                              if dist else "this GPU's plan")},
    }
    if rank == 0 and not args.no_cpu:
        try:
            rate, cn, cdt = cpu_reference_rate(args, args.cpu_seconds)
            line["cpu_baseline"] = {
                "value": rate / 1e6, "unit": METRIC, "cores": os.cpu_count(), "kind": "port",
                "cpu_model": cpu_model(),
                "sample": "%d realisations of the same scene in %.1f s (OpenMP, all cores)"
                          % (cn, cdt)}
        except Exception as exc:
            line["cpu_baseline"] = {"value": None, "unit": METRIC, "cores": os.cpu_count(),
                                    "kind": "port", "cpu_model": cpu_model(),
                                    "sample": "failed: %s" % exc}
    del e
    s.close()
    if args.config == "field" and args.heliostats == 1000 and not args.no_suns:
        # The other half of the metric: time to 0.1 % SE on absorbed power
        # for the 256 suns, batched against plain per-sun launches
        r = suns_comparison(args, lib, opt, stream, sp, flush, dist, local, rank, world,
                            min(args.steps, 3), min(args.warmup, 3))
        line["time_to_0.1pct_se"] = {
            "workload": SUNS, "suns": r["suns"], "paths": r["paths"],
            "steps": min(args.steps, 3), "warmup": min(args.warmup, 3),
            "batched_s": r["time_to_0.1pct_se_s"]["batched"],
            "batched_host_built_scenes_s": r["time_to_0.1pct_se_s"]["batched_host_built_scenes"],
            "plain_fp32_plan_loop_s": r["time_to_0.1pct_se_s"]["plain_plan_loop"],
            "plain_fp32_ssol_solve_loop_s": r["time_to_0.1pct_se_s"]["ssol_solve_loop"],
            "speedup_vs_plan_loop": r["speedup_batched_vs_plain_plan_loop"],
            "speedup_vs_ssol_solve_loop": r["speedup_batched_vs_ssol_solve_loop"],
            "from_scratch_s": r["time_to_0.1pct_se_from_scratch_s"],
            "speedup_from_scratch_vs_plan_loop": r["speedup_from_scratch_vs_plain_plan_loop"],
            "speedup_from_scratch_vs_plan_loop_device_bvh":
                r["speedup_from_scratch_vs_plain_plan_loop_device_bvh"],
            "speedup_from_scratch_vs_ssol_solve_loop":
                r["speedup_from_scratch_vs_ssol_solve_loop"],
            "suns_reaching_0.1pct_se": r["reached"],
            "batched_mpaths_s": r["paths"] / r["per_step_batched_ms"] / 1e3,
            "clocks": r["clocks"],
            "arms": "batched: every sun in one persistent launch replayed from a CUDA "
                    "graph, items built on the device from one snapshot (tracking batch; "
                    "CUDA events); batched_host_built_scenes: the same launch over 256 "
                    "host snapshots; plain_fp32_plan_loop: one plain FP32 plan "
                    "launch per sun, scenes resident (CUDA events); "
                    "plain_fp32_ssol_solve_loop: one ssol_solve per sun (wall clock); "
                    "from_scratch: pilot of 1e5 per sun, read-back, then the rest, "
                    "set-up included (wall clock)"}
    if (args.config == "field" and args.heliostats == 1000 and not args.no_suns
            and not args.no_others and world == 1 and rank == 0):
        line["other_configs"] = other_configs()
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


BVH_CHOICES = {"auto": 0, "sah": 1, "lbvh": 2}


def counted_stats(lib, s, opt, n, seed, sp):
    """Stats of one launch of n paths with the work counters on, with the
    launch shape and builder of `opt`."""
    import pyssol as P
    o = P.options(opt.precision, block_size=opt.block_size, waves=opt.waves,
                  leaf=opt.bvh_leaf_size, min_blocks=opt.min_blocks_per_sm,
                  bvh=opt.bvh_builder, count=1)
    plan = P.C.c_void_p()
    lib.call("ssol_b200_plan_create", s.scn, P.C.byref(o), P.C.byref(plan))
    rng = s.rng(seed=seed)
    lib.call("ssol_b200_plan_launch", plan, rng, 0, n, sp)
    est = P.C.c_void_p()
    res = lib.raw("ssol_b200_plan_finish", plan, rng, n, 0, sp, P.C.byref(est))
    st = P.Estimator(s, est, res).stats()
    lib.raw("ssol_b200_plan_ref_put", plan)
    return st


def bvh_builders(lib, s, opt, n, stream, sp, flush):
    """The two BVH builders on this scene, outside the timed region: plan
    creation wall time (snapshot, tree, upload; median of 3), device
    Mpaths/s of 2 launches of n paths after 1 warm-up (CUDA events, L2
    flushed between launches; the kernel variant with work counters, for the
    node visits per path), the tree's depth, and an ssol_solve_ex of 1e6
    paths end to end (median of 5), where the build is a large part of the
    call."""
    import torch
    import pyssol as P
    out = {}
    for name, b in (("sah_host", P.BVH_SAH), ("lbvh_device", P.BVH_LBVH)):
        o = P.options(opt.precision, block_size=opt.block_size, waves=opt.waves,
                      leaf=opt.bvh_leaf_size, min_blocks=opt.min_blocks_per_sm, bvh=b,
                      count=1)
        create = []
        for k in range(3):
            plan = P.C.c_void_p()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            lib.call("ssol_b200_plan_create", s.scn, P.C.byref(o), P.C.byref(plan))
            torch.cuda.synchronize()
            create.append((time.perf_counter() - t0) * 1e3)
            if k < 2:
                lib.raw("ssol_b200_plan_ref_put", plan)
        rng = s.rng(seed=123)
        lib.call("ssol_b200_plan_launch", plan, rng, 0, n, sp)
        lib.call("ssol_b200_plan_reset", plan, sp)
        if flush is not None:
            flush.zero_()
        ms = 0.0
        for k in range(2):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            lib.call("ssol_b200_plan_launch", plan, rng, (1 + k) * n, n, sp)
            e1.record(stream)
            if flush is not None:
                flush.zero_()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
        est = P.C.c_void_p()
        res = lib.raw("ssol_b200_plan_finish", plan, rng, 2 * n, 0, sp, P.C.byref(est))
        e = P.Estimator(s, est, res)
        st = e.stats()
        del e
        lib.raw("ssol_b200_plan_ref_put", plan)
        solve = []
        for k in range(5):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ek = s.solve(1_000_000, seed=k, options=o)
            solve.append((time.perf_counter() - t0) * 1e3)
            del ek
        out[name] = {"plan_create_ms": sorted(create)[1],
                     "mpaths_s": 2 * n / (ms * 1e-3) / 1e6,
                     "node_visits_per_path": st["node_visits"] / max(1, st["paths"]),
                     "depth": st["bvh_depth"], "nodes": st["bvh_nodes"],
                     "built_on_device": bool(st["bvh_device"]),
                     "ssol_solve_ex_1e6_ms": sorted(solve)[2]}
    return out


# The other workloads of the repo, measured by the default line too (each in
# a child process of its own, as `bench.py --config X` would run it, with
# 3 warm-up and 3 timed steps)
OTHER_CONFIGS = (
    ("beamdown", ["--config", "beamdown", "--steps", "3", "--warmup", "3", "--no-cpu"]),
    ("adjoint", ["--config", "adjoint", "--steps", "3", "--warmup", "3", "--no-cpu"]),
    ("draft", ["--config", "draft", "--steps", "3", "--warmup", "3", "--no-cpu"]),
    ("pt", ["--config", "pt", "--steps", "3", "--warmup", "3", "--no-cpu"]),
)


def other_configs():
    """Run OTHER_CONFIGS one after the other; per config the key figures of
    its JSON line (or why it has none)."""
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "LOCAL_WORLD_SIZE",
                        "MASTER_ADDR", "MASTER_PORT", "GROUP_RANK")
           and not k.startswith("TORCHELASTIC")}
    out = {}
    for name, flags in OTHER_CONFIGS:
        try:
            proc = subprocess.run([sys.executable, os.path.abspath(__file__)] + flags,
                                  capture_output=True, text=True, timeout=900, env=env)
            lines = [ln for ln in proc.stdout.splitlines() if ln.startswith("{")]
            if proc.returncode != 0 or not lines:
                out[name] = {"failed": "exit %d: %s" % (proc.returncode,
                                                        proc.stderr.strip()[-300:])}
                continue
            d = json.loads(lines[-1])
            r = {"workload": (d.get("config") or {}).get("workload"),
                 "value": d.get("value"), "unit": d.get("unit"),
                 "ms_per_step": d.get("ms_per_step"), "steps": d.get("steps"),
                 "warmup": d.get("warmup"), "dtype": d.get("dtype"),
                 "e2e": (d.get("e2e") or {}).get("value"),
                 "roofline_frac": (d.get("roofline") or {}).get("frac"),
                 "clocks": d.get("clocks")}
            if d.get("precision_vs_fp64"):
                r["precision_vs_fp64_max_rel_diff"] = d["precision_vs_fp64"].get(
                    "max_abs_rel_diff")
            if d.get("fd_check"):
                r["fd_check"] = d["fd_check"]
            if d.get("bvh_builders"):
                r["bvh_builders"] = d["bvh_builders"]
            out[name] = r
        except Exception as exc:
            out[name] = {"failed": str(exc)}
    return out


SUNS = ("256 suns (16 elevations 5-85 deg x 16 azimuths, DNI U[300,1000]) over the "
        "1000-heliostat field re-aimed per sun; per-sun budgets = realisations for 0.1% "
        "relative SE on absorbed power (from a pilot of log-U[1e5,1e7] budgets)")


def suns_comparison(args, lib, opt, stream, sp, flush, dist, local, rank, world,
                    steps, warmup):
    """Batched multi-sun form against plain per-sun launches, as a dict.

    Pilot: one batched launch with the seeded log-uniform budgets gives each
    sun's relative SE on absorbed power, hence the realisations n_i it needs
    for 0.1% (SE ~ 1/sqrt(n)). Timed, for the same n_i: (a) the batched
    launch (all suns in one persistent kernel replayed from a CUDA graph),
    (b) a loop of plain plan launches, one per sun, scenes resident in HBM,
    (c) end to end through the public API, per step: batch create (scene
    build and upload), launch, finish (tally read-back and estimators);
    and (d) the reference user's loop of one ssol_solve per sun. From
    scratch (e): each approach runs a pilot of 1e5 realisations per sun,
    reads its estimates back and traces what each sun still needs."""
    import torch
    import pyssol as P
    import workloads as W
    grid = W.sun_grid()
    if args.suns:
        # evenly spaced subset of the 256 suns (small cases, profiling)
        step = max(1, len(grid) // args.suns)
        grid = grid[::step][:args.suns]
    suns = shard_suns(grid, rank, world)
    built = W.batched_fields(lib, suns, n_helio=args.heliostats)
    scenes = [b[0] for b in built]
    rng = scenes[0].rng(seed=args.seed)
    # The batched form: one snapshot of the field, its heliostats re-aimed
    # per sun and its BVH refitted on the device (a tracking batch)
    base, hb = W.heliostat_field(lib, n_helio=args.heliostats)
    track_in = W.tracking_inputs(hb, suns)

    def tracking_batch():
        return P.Batch.tracking(base, *track_in, opts=opt)

    # pilot
    pilot = tracking_batch()
    pilot.launch(rng, [sn["budget"] for sn in suns], sp)
    ests = pilot.finish(rng, 0, sp)
    target = 1e-3
    need = []
    for sn, e in zip(suns, ests):
        a = e.globals()["absorbed_by_receivers"]
        rse = a[2] / a[0] if a[0] > 0 else 1.0
        need.append(int(min(max(sn["budget"] * (rse / target) ** 2, 1e5), 1e8)))
    del ests
    pilot.close()
    n_total = sum(need)

    def timed(step):
        for w in range(warmup):
            step()
            flush.zero_()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        for k in range(steps):
            ev[k][0].record(stream)
            step()
            ev[k][1].record(stream)
            flush.zero_()
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in ev)
        if dist:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t[0])
        return ms

    # (a) batched: the tracking batch, and a batch of the host-built scenes
    batch = tracking_batch()
    clocks = Clocks(local)
    clocks.start()
    ms_batched = timed(lambda: batch.launch(rng, need, sp))
    clk = clocks.stop()
    sbatch = P.Batch(lib, scenes, opt)
    ms_scene_batch = timed(lambda: sbatch.launch(rng, need, sp))
    sbatch.close()
    ests = batch.finish(rng, 0, sp)
    # counters and scene bytes are batch-wide (every item's estimator carries
    # them); tally bytes are per item
    bstats = ests[0].stats()
    tally_bytes = sum(e.stats()["tally_bytes"] for e in ests)
    reached = sum(1 for e in ests if e.globals()["absorbed_by_receivers"][2]
                  <= target * e.globals()["absorbed_by_receivers"][0] * 1.05)
    del ests
    batch.close()
    # The work per launch for the roofline model: the timed launches leave
    # the work counters out (the library's default); one counted launch of
    # the same batch, outside the timed region, gives them
    o_c = P.options(opt.precision, block_size=opt.block_size, waves=opt.waves,
                    leaf=opt.bvh_leaf_size, min_blocks=opt.min_blocks_per_sm,
                    bvh=opt.bvh_builder, count=1)
    cb = P.Batch.tracking(base, *track_in, opts=o_c)
    cb.launch(rng, need, sp)
    ces = cb.finish(rng, 0, sp)
    cstats = ces[0].stats()
    del ces
    cb.close()

    # (b) plain plan launches, one per sun
    plans = []
    for sc in scenes:
        pl = P.C.c_void_p()
        lib.call("ssol_b200_plan_create", sc.scn, P.C.byref(opt), P.C.byref(pl))
        plans.append(pl)

    def plain_step():
        for pl, n in zip(plans, need):
            lib.call("ssol_b200_plan_launch", pl, rng, 0, n, sp)
    ms_plain = timed(plain_step)
    for pl in plans:
        lib.raw("ssol_b200_plan_ref_put", pl)

    # (c) end to end through the batch API, and (d) one ssol_solve per sun
    h2d = bstats["scene_bytes"]
    d2h = tally_bytes
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_steps = max(1, min(steps, 2))
    for k in range(e2e_steps):
        b = tracking_batch()
        b.launch(rng, need, sp)
        es = b.finish(rng, 0, sp)
        del es
        b.close()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    t0 = time.perf_counter()
    for sc, n in zip(scenes, need):
        e = sc.solve(n, rng=rng, options=opt)
        del e
    solve_loop_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s, solve_loop_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s, solve_loop_s = float(t[0]), float(t[1])
        tot = torch.tensor([float(n_total)], device="cuda")
        dist.all_reduce(tot)
        n_all = float(tot[0])
    else:
        n_all = float(n_total)

    # (e) from scratch: each approach runs a pilot of 1e5 realisations per
    # sun, reads its estimates back, and traces the realisations each sun
    # still needs for 0.1 % SE; wall clock, scene snapshots included. The
    # plain loop does this sun by sun, as a caller running every sun to a
    # target SE with the plain kernel must.
    budgets = [100000 for _ in suns]

    def needed_g(g, done_n):
        a = g["absorbed_by_receivers"]
        rse = a[2] / a[0] if a[0] > 0 else 1.0
        return int(min(max(done_n * (rse / target) ** 2, done_n), 1e8))

    def needed(est, done_n):
        return needed_g(est.globals(), done_n)

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bt = tracking_batch()
    bt.launch(rng, budgets, sp)
    # the pilot needs each sun's absorbed-power SE only: the per-item global
    # estimates, read without building estimators
    more = [needed_g(g, b) - b for g, b in zip(bt.globals(sp), budgets)]
    bt.launch(rng, more, sp)
    es = bt.finish(rng, 0, sp)
    # time to the results: the estimators exist; releasing the batch is not
    # part of it (the per-sun loops release each sun's plan before the next)
    scratch_batched = time.perf_counter() - t0
    del es
    bt.close()
    def plain_from_scratch(o):
        t0 = time.perf_counter()
        for sc, b in zip(scenes, budgets):
            pl = P.C.c_void_p()
            lib.call("ssol_b200_plan_create", sc.scn, P.C.byref(o), P.C.byref(pl))
            lib.call("ssol_b200_plan_launch", pl, rng, 0, b, sp)
            est = P.C.c_void_p()
            lib.raw("ssol_b200_plan_finish", pl, rng, b, 0, sp, P.C.byref(est))
            e = P.Estimator(sc, est, 0)
            tot = needed(e, b)
            del e
            if tot > b:
                lib.call("ssol_b200_plan_launch", pl, rng, b, tot - b, sp)
                est = P.C.c_void_p()
                lib.raw("ssol_b200_plan_finish", pl, rng, tot, 0, sp, P.C.byref(est))
                lib.raw("ssol_estimator_ref_put", est)
            lib.raw("ssol_b200_plan_ref_put", pl)
        return time.perf_counter() - t0

    scratch_plain = plain_from_scratch(opt)
    # the same loop with each sun's tree built on the device
    opt_lbvh = P.options(opt.precision, block_size=opt.block_size, waves=opt.waves,
                         leaf=opt.bvh_leaf_size, min_blocks=opt.min_blocks_per_sm,
                         bvh=P.BVH_LBVH)
    scratch_plain_lbvh = plain_from_scratch(opt_lbvh)
    t0 = time.perf_counter()
    for sc, b in zip(scenes, budgets):
        r1 = sc.rng(seed=args.seed + 5)
        e = sc.solve(b, rng=r1, options=opt)
        tot = needed(e, b)
        if tot > b:
            state = P.C.c_void_p()
            lib.call("ssol_estimator_get_rng_state", e.h, P.C.byref(state))
            e2 = sc.solve(tot - b, rng=state, options=opt)
            del e2
        del e
    scratch_solve = time.perf_counter() - t0
    for sc in scenes:
        sc.close()
    base.close()

    per_step_b = ms_batched / steps
    per_step_p = ms_plain / steps
    agg = {k: cstats[k] for k in ("rays", "node_visits", "triangle_tests",
                                  "quadric_tests", "bounces", "paths")}
    return {
        "suns": len(suns) * world, "paths": int(n_all), "n_total_rank": n_total,
        "per_step_batched_ms": per_step_b, "per_step_plain_ms": per_step_p,
        "agg": agg, "launches": 1, "clocks": clk, "h2d": h2d, "d2h": d2h,
        "e2e_s": e2e_s, "reached": reached,
        "time_to_0.1pct_se_s": {"batched": per_step_b * 1e-3,
                                "batched_host_built_scenes": ms_scene_batch / steps * 1e-3,
                                "plain_plan_loop": per_step_p * 1e-3,
                                "ssol_solve_loop": solve_loop_s,
                                "batch_api_end_to_end": e2e_s},
        "time_to_0.1pct_se_from_scratch_s": {
            "batched": scratch_batched, "plain_plan_loop_per_sun": scratch_plain,
            "plain_plan_loop_per_sun_device_bvh": scratch_plain_lbvh,
            "ssol_solve_loop_per_sun": scratch_solve,
            "what": "pilot of 1e5 per sun + read-back + the rest, per approach, "
                    "scene snapshots included (batched: one snapshot, re-aimed per "
                    "sun on the device; the loops: one snapshot per sun); the "
                    "per-sun loops synchronise once per pilot"},
        "speedup_from_scratch_vs_plain_plan_loop": scratch_plain / scratch_batched,
        "speedup_from_scratch_vs_plain_plan_loop_device_bvh":
            scratch_plain_lbvh / scratch_batched,
        "speedup_from_scratch_vs_ssol_solve_loop": scratch_solve / scratch_batched,
        "speedup_batched_vs_plain_plan_loop": per_step_p / per_step_b,
        "speedup_batched_vs_ssol_solve_loop": solve_loop_s / (per_step_b * 1e-3),
    }


def run_suns(args):
    """The batched multi-sun line (see suns_comparison)."""
    import torch
    import pyssol as P
    import workloads as W
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    lib = P.load_product()
    opt = P.options(P.FP64 if args.fp64 else P.FP32, block_size=args.block,
                    waves=args.waves, leaf=args.leaf, min_blocks=args.minb,
                    bvh=BVH_CHOICES[args.bvh])
    if args.autotune:
        s, h = W.heliostat_field(lib, n_helio=args.heliostats, elevation=45.0)
        opt, _ = P.autotune(s, args.autotune_paths, opt, seed=args.seed + 77)
        s.close()
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = P.C.c_void_p(stream.cuda_stream)
    flush = torch.empty(max(1, args.flush_mib) * 1024 * 1024 // 4, dtype=torch.float32,
                        device="cuda")
    r = suns_comparison(args, lib, opt, stream, sp, flush, dist, local, rank, world,
                        args.steps, args.warmup)
    per_step_b = r["per_step_batched_ms"]
    value = r["paths"] / (per_step_b * 1e-3) / 1e6
    peaks = measured_peaks()
    nsm = torch.cuda.get_device_properties(local).multi_processor_count
    sm_mhz = peaks.get("sm_max_mhz", 1965.0)
    fp32_peak = nsm * 128 * 2 * sm_mhz * 1e6 / 1e12
    # the counters cover the warm-up and timed launches of the batch
    achieved = flops_per_run(r["agg"]) / r["launches"] / (per_step_b * 1e-3) / 1e12
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step_b,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64" if args.fp64 else "f32",
        "data": "synthetic (seeded sun grid, DNI and budgets)",
        "config": {"workload": SUNS, "suns": r["suns"],
                   "paths_per_step": r["paths"],
                   "l2": "flushed: 256 MiB write between steps",
                   "parallelism": "sun slots per GPU" if world > 1 else "1 GPU",
                   "launch": {"block": opt.block_size,
                              "blocks_per_sm_budget": opt.min_blocks_per_sm,
                              "waves": opt.waves, "bvh_leaf": opt.bvh_leaf_size,
                              "autotuned": bool(args.autotune)}},
        "e2e": {"value": r["paths"] / r["e2e_s"] / 1e6, "unit": METRIC,
                "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"],
                "timing": "wall clock: batch create + launch + finish per step"},
        # batched launches of 2^22 to 2^29 realisations run the coherent
        # order's presort (count, scan, scatter) before the batched kernel
        "gpu_launches": args.steps * (4 if (1 << 22) <= r["n_total_rank"] <= (1 << 29) else 1),
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak,
                     "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                     "traffic": BATCH_DRAM_BYTES_PER_PATH * r["n_total_rank"],
                     "traffic_source": "ncu dram__bytes_read+write of the batched kernel on "
                                       "32 suns (3.2e7 paths), scaled to this rank's paths per launch",
                     "work_model": "as the field line"},
        "clocks": r["clocks"],
        "suns_reaching_0.1pct_se": r["reached"],
    }
    for k in ("time_to_0.1pct_se_s", "time_to_0.1pct_se_from_scratch_s",
              "speedup_from_scratch_vs_plain_plan_loop",
              "speedup_from_scratch_vs_plain_plan_loop_device_bvh",
              "speedup_from_scratch_vs_ssol_solve_loop",
              "speedup_batched_vs_plain_plan_loop", "speedup_batched_vs_ssol_solve_loop"):
        line[k] = r[k]
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


ADJOINT = ("aim gradients (ssol_solve_adjoint) on the 1000-heliostat field: 2000 aim "
           "angles (2 per heliostat), initial aim offsets uniform in +-2 mrad (seeded), "
           "objectives first-bounce absorbed power and spillage "
           "sum_c (map - uniform target)^2 on a 64x64 map of the 12x12 receiver")
AIM_OFFSET = 2e-3  # rad, half-width of the seeded initial aim offsets


def run_adjoint(args):
    """Adjoint of the field's first-bounce flux map w.r.t. every heliostat's two
    aim angles. value: Mpaths/s of the two replayed passes (CUDA-event time of
    the kernels, scene resident); e2e: wall clock of the synchronous call
    (snapshot, upload, both passes, read-back). Then central finite differences
    with common random numbers on 32 seeded random parameters, at h = 1e-4
    and 1e-3 rad, and the relative error of the adjoint against them (the
    bias of the shadowing and blocking terms it leaves out; its receiver-edge
    term is smoothed over half a map cell)."""
    import random
    import torch
    import pyssol as P
    import workloads as W
    import adjoint as A
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    lib = P.load_product()
    s, h = W.heliostat_field(lib, n_helio=args.heliostats)
    lower, upper, nx, ny = (-6.0, -6.0), (6.0, 6.0), 64, 64
    n = args.paths
    # initial aim offsets: every heliostat turned by seeded uniform angles in
    # +-AIM_OFFSET about its two local axes; gradients and finite differences
    # are taken about this configuration
    aims = A.AimField(s, h["heliostats"], h["transforms"], h["receiver"], lower, upper,
                      nx, ny, 0.0, n)
    rnd0 = random.Random(args.seed + 5)
    transforms = []
    for i in range(len(h["heliostats"])):
        xf = aims.offset_transform(i, rnd0.uniform(-AIM_OFFSET, AIM_OFFSET),
                                   rnd0.uniform(-AIM_OFFSET, AIM_OFFSET))
        lib.call("ssol_instance_set_transform", h["heliostats"][i], P._transform(xf))
        transforms.append(xf)
    opt = P.options(P.FP64 if args.fp64 else P.FP32)
    base = A.solve_adjoint(s, h["heliostats"], h["receiver"], lower, upper, nx, ny, 0.0,
                           n, seed=args.seed, options=opt, want_map=True)
    target = sum(base["map"]) / len(base["map"])
    for w in range(args.warmup):
        A.solve_adjoint(s, h["heliostats"], h["receiver"], lower, upper, nx, ny, target,
                        n, seed=args.seed + 1 + w, options=opt)
    clocks = Clocks(local)
    clocks.start()
    kms, t0 = 0.0, time.perf_counter()
    cnt = {}
    for k in range(args.steps):
        r = A.solve_adjoint(s, h["heliostats"], h["receiver"], lower, upper, nx, ny, target,
                            n, seed=args.seed + 100 + k, options=opt)
        kms += r["kernel_ms"]
        for key, v in r["counters"].items():
            cnt[key] = cnt.get(key, 0) + v
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    value = args.steps * n / (kms * 1e-3) / 1e6
    # FP32 work model of the field line; each realisation is sampled in both
    # passes and each unshadowed one casts a reflected ray (rays - samples)
    passes = 2
    samples = passes * args.steps * n
    reflected = max(0, cnt["rays"] - samples)
    flops = (20 * 2 * cnt["node_visits"] + 55 * cnt["triangle_tests"]
             + 90 * cnt["quadric_tests"] + 150 * reflected + 120 * samples)
    achieved = flops / (kms * 1e-3) / 1e12
    nsm = torch.cuda.get_device_properties(local).multi_processor_count
    fp32_peak = nsm * 128 * 2 * measured_peaks().get("sm_max_mhz", 1965.0) * 1e6 / 1e12
    e2e = args.steps * n / wall / 1e6

    fd = {}
    if args.fd_params > 0:
        field = A.AimField(s, h["heliostats"], transforms, h["receiver"], lower, upper,
                           nx, ny, target, args.fd_paths, seed=args.seed + 7, options=opt)
        rnd = random.Random(args.seed)
        params = [(rnd.randrange(len(h["heliostats"])), rnd.randrange(2))
                  for _ in range(args.fd_params)]
        for step in (1e-4, 1e-3):
            _, rows = A.finite_difference_check(field, params, h=step)
            out = {}
            for key in ("spillage", "absorbed"):
                a = [row["adjoint_" + key] for row in rows]
                b = [row["fd_" + key] for row in rows]
                nb = math.sqrt(sum(x * x for x in b)) or 1.0
                na = math.sqrt(sum(x * x for x in a)) or 1.0
                out[key] = {"rel_l2_error": math.sqrt(sum((x - y) ** 2 for x, y in zip(a, b)))
                            / nb,
                            "cosine": sum(x * y for x, y in zip(a, b)) / (na * nb)}
            fd["h=%g" % step] = out
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": kms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.fp64 else "f32",
        "data": "synthetic (seeded generator, no public scene)",
        "config": {"workload": ADJOINT, "paths_per_step": n, "parameters": 2 * len(
            h["heliostats"]), "passes": 2, "map": "64x64 over 12x12, bilinear splat",
            "l2": "not flushed (scene < 2 MB; the map and gradients are rewritten)"},
        "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": None,
                "d2h_bytes_per_step": (nx * ny + 4 * len(h["heliostats"])) * 8,
                "timing": "wall clock around the synchronous ssol_solve_adjoint"},
        "gpu_launches": 2 * args.steps,
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak,
                     "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                     "traffic": ADJOINT_DRAM_BYTES_PER_PATH * n / passes,
                     "traffic_source": "ncu dram__bytes_read+write of both passes on 4e6 "
                                       "paths, scaled to the step's paths, per launch "
                                       "(mean of the two passes)",
                     "peak_source": "SMs x 128 FP32 lanes x 2 x measured max SM clock "
                                    "(MEASURED_PEAKS.json sm_max_mhz)",
                     "work_model": "20/slab x2 per node + 55/triangle + 90/quadric + "
                                   "150/reflected ray + 120/sample per pass (counted on "
                                   "device)",
                     "counters_per_path": {k: v / (args.steps * n) for k, v in cnt.items()}},
        "objective": {"absorbed_W": base["absorbed"], "spillage": base["spillage"],
                      "target_W_m2": target},
        "fd_check": {"params": args.fd_params, "paths": args.fd_paths,
                     "common_random_numbers": True, **fd},
        "clocks": clk,
    }
    print(json.dumps(line))


DRAW = ("{kind}: the 1000-heliostat field (mirrors Beckmann 2 mrad, 12x12 receiver on a "
        "100 m tower, pillbox sun el 30 az 180) over a 4x4 km matte ground (reflectivity "
        "0.3), seen from (0, -60, 170) toward (0, 280, 0), 75 deg horizontal field of view, "
        "{w}x{h} pixels, {spp} samples per pixel, sky radiance 0.1 above +z")
DRAW_CAMERA = ((0.0, -60.0, 170.0), (0.0, 280.0, 0.0), (0.0, 0.0, 1.0), math.radians(75.0))


def draw_scene(lib, args):
    import pyssol as P
    import workloads as W
    s, h = W.heliostat_field(lib, n_helio=args.heliostats)
    ground = s.matte(0.3)
    s.instance(s.object([(s.rectangle(2000, 2000), ground, ground)]),
               P.transform_from(None, (0.0, 0.0, -0.5)), sample=0)
    pos, tgt, up, fov = DRAW_CAMERA
    cam = s.camera(pos, tgt, up, fov=fov, ratio=args.width / args.height)
    desc = DRAW.format(kind="ssol_draw_pt path tracing" if args.config == "pt"
                       else "ssol_draw_draft", w=args.width, h=args.height, spp=args.spp)
    return s, cam, desc


def oracle_draw_rate(args, seconds):
    """Oracle camera samples/s on all host cores: the same camera on a
    reduced image whose samples take about `seconds`."""
    import pyssol as P
    lib = P.Lib(ORACLE_LIB)
    s, cam, _ = draw_scene(lib, args)
    kind = args.config
    img = P.C.c_void_p()
    lib.call("ssol_image_create", s.dev, P.C.byref(img))

    def run(w, hh, spp):
        lib.call("ssol_image_setup", img, w, hh, P.PIXEL_DOUBLE3)
        wr = P.WRITE_PIXELS(("ssol_image_write", lib.dll))
        t = time.perf_counter()
        if kind == "draft":
            lib.call("ssol_draw_draft", s.scn, cam, w, hh, spp, wr, img)
        else:
            lib.call("ssol_draw_pt", s.scn, cam, w, hh, spp, (P.C.c_double * 3)(0, 0, 1),
                     wr, img)
        return time.perf_counter() - t

    probe_w, probe_h = max(16, args.width // 16), max(9, args.height // 16)
    dt = run(probe_w, probe_h, args.spp)
    rate = probe_w * probe_h * args.spp / dt
    scale = min(1.0, math.sqrt(rate * seconds / (args.width * args.height * args.spp)))
    w, hh = max(16, int(args.width * scale)), max(9, int(args.height * scale))
    dt = run(w, hh, args.spp)
    lib.call("ssol_image_ref_put", img)
    s.close()
    return w * hh * args.spp / dt, w, hh, dt


def run_draw(args):
    """The preview renderers. value: camera samples/s of the draw kernel (its
    CUDA-event time, scene resident, L2 flushed between steps); e2e: wall
    clock of the public ssol_draw_* call with ssol_image_write as the writer
    (snapshot, upload, kernel, image read-back, tiles to the host image)."""
    import torch
    import pyssol as P
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    lib = P.load_product()
    s, cam, desc = draw_scene(lib, args)
    opt = P.options(P.FP64 if args.fp64 else P.FP32)
    W_, H_, spp = args.width, args.height, args.spp
    buf = torch.empty((H_, W_, 3), dtype=torch.float64, device="cuda")
    flush = torch.empty(max(1, args.flush_mib) * 1024 * 1024 // 4, dtype=torch.float32,
                        device="cuda")
    seed = args.seed

    def step(k):
        return s.draw_device(args.config, cam, W_, H_, spp, buf.data_ptr(), up=(0, 0, 1),
                             seed=seed + k, options=opt)

    for w in range(args.warmup):
        step(w)
        if args.flush_mib:
            flush.zero_()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    kms, totals = 0.0, {}
    for k in range(args.steps):
        st = step(args.warmup + k)
        kms += st.kernel_ms
        for f in ("rays", "node_visits", "triangle_tests", "quadric_tests", "bounces",
                  "paths"):
            totals[f] = totals.get(f, 0) + getattr(st, f)
        scene_bytes = st.scene_bytes
        if args.flush_mib:
            flush.zero_()
            torch.cuda.synchronize()
    clk = clocks.stop()
    samples = W_ * H_ * spp
    value = args.steps * samples / (kms * 1e-3) / 1e6

    e2e = None
    if not args.no_e2e:
        img = P.C.c_void_p()
        lib.call("ssol_image_create", s.dev, P.C.byref(img))
        lib.call("ssol_image_setup", img, W_, H_, P.PIXEL_DOUBLE3)
        wr = P.WRITE_PIXELS(("ssol_image_write", lib.dll))
        up = (P.C.c_double * 3)(0, 0, 1)

        def public():
            if args.config == "draft":
                lib.call("ssol_draw_draft", s.scn, cam, W_, H_, spp, wr, img)
            else:
                lib.call("ssol_draw_pt", s.scn, cam, W_, H_, spp, up, wr, img)
        public()
        t0 = time.perf_counter()
        e2e_steps = max(1, min(args.steps, 3))
        for k in range(e2e_steps):
            public()
        dt = time.perf_counter() - t0
        e2e = e2e_steps * samples / dt / 1e6
        lib.call("ssol_image_ref_put", img)

    peaks = measured_peaks()
    nsm = torch.cuda.get_device_properties(local).multi_processor_count
    sm_mhz = peaks.get("sm_max_mhz", 1965.0)
    fp32_peak = nsm * 128 * 2 * sm_mhz * 1e6 / 1e12
    achieved = flops_per_run(totals) / (kms * 1e-3) / 1e12 if kms > 0 else 0.0
    unit = "Msamples/s"
    line = {
        "metric": unit, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": kms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.fp64 else "f32",
        "data": "synthetic (seeded generator, no public scene)",
        "config": {"workload": desc, "samples_per_step": samples,
                   "l2": ("flushed: %d MiB write between steps (scene < 2 MB, image %.0f MB)"
                          % (args.flush_mib, W_ * H_ * 24 / 1e6)
                          if args.flush_mib else "not flushed (profiling run)")},
        "e2e": {"value": e2e, "unit": unit, "h2d_bytes_per_step": scene_bytes,
                "d2h_bytes_per_step": W_ * H_ * 24,
                "timing": "wall clock around the synchronous ssol_draw_* call"},
        "gpu_launches": args.steps,
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak,
                     "unit": "TFLOP/s", "frac": achieved / fp32_peak if fp32_peak else None,
                     "traffic": None,
                     "peak_source": "SMs x 128 FP32 lanes x 2 x measured max SM clock "
                                    "(MEASURED_PEAKS.json sm_max_mhz)",
                     "work_model": "20/slab x2 per node + 55/triangle + 90/quadric + "
                                   "150/bounce + 120/sample (counted on device)",
                     "counters_per_sample": {k: totals[k] / max(1, totals["paths"]) for k in
                                             ("rays", "node_visits", "triangle_tests",
                                              "quadric_tests", "bounces")},
                     "kernel_ms": kms},
        "clocks": clk,
        "image_mean": float(buf.mean()),
    }
    if not args.no_cpu:
        try:
            rate, cw, ch, cdt = oracle_draw_rate(args, args.cpu_seconds)
            line["cpu_baseline"] = {
                "value": rate / 1e6, "unit": unit, "cores": os.cpu_count(), "kind": "port",
                "sample": "%dx%d pixels x %d samples of the same view in %.1f s (OpenMP, "
                          "all cores)" % (cw, ch, spp, cdt)}
        except Exception as exc:
            line["cpu_baseline"] = {"value": None, "unit": unit, "cores": os.cpu_count(),
                                    "kind": "port", "sample": "failed: %s" % exc}
    print(json.dumps(line))
    s.close()


def run_draw_reference(args):
    """The oracle's renderer on the host cores, each step a bounded sample
    (a reduced image of the same view)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    rates = []
    for k in range(args.warmup + args.steps):
        rate, cw, ch, cdt = oracle_draw_rate(args, args.ref_step_seconds)
        if k >= args.warmup:
            rates.append((rate, cw, ch, cdt))
    total_s = sum(r[3] for r in rates)
    total = sum(r[0] * r[3] for r in rates)
    value = total / total_s / 1e6
    unit = "Msamples/s"
    s_desc = DRAW.format(kind="ssol_draw_pt path tracing" if args.config == "pt"
                         else "ssol_draw_draft", w=args.width, h=args.height, spp=args.spp)
    line = {
        "impl": "reference", "metric": unit, "value": value, "unit": unit,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": s_desc, "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": unit, "cores": os.cpu_count(), "kind": "port",
                         "sample": "%dx%d pixels x %d samples per step" % (
                             rates[0][1], rates[0][2], args.spp)},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--config", default="field",
                   choices=["field", "mirror", "beamdown", "suns", "adjoint", "draft",
                            "pt"])
    p.add_argument("--width", type=int, default=1920)
    p.add_argument("--height", type=int, default=1080)
    p.add_argument("--spp", type=int, default=None,
                   help="samples per pixel of the draw configs (draft 4, pt 16)")
    p.add_argument("--fd-params", type=int, default=32)
    p.add_argument("--fd-paths", type=int, default=100_000_000)
    p.add_argument("--heliostats", type=int, default=1000)
    p.add_argument("--suns", type=int, default=0,
                   help="suns config: evenly spaced subset of this many suns (0: all 256)")
    p.add_argument("--paths", type=int, default=None,
                   help="realisations per step (field 1e8, beamdown 2e8, mirror 1e6)")
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--fp64", action="store_true")
    p.add_argument("--block", type=int, default=256)
    p.add_argument("--waves", type=int, default=1)
    p.add_argument("--leaf", type=int, default=0)
    p.add_argument("--minb", type=int, default=0)
    p.add_argument("--no-autotune", dest="autotune", action="store_false",
                   help="use --block/--minb/--waves/--leaf as given")
    p.add_argument("--autotune-paths", type=int, default=4_000_000)
    p.add_argument("--flush-mib", type=int, default=256,
                   help="L2 flush buffer written between steps (profiling: 0)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-fp64-check", action="store_true",
                   help="skip the FP32 vs all-FP64 comparison of the field configs")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--bvh", default="auto", choices=sorted(BVH_CHOICES),
                   help="BVH builder of the solves (auto: by solve size for ssol_solve, "
                        "host SAH for plans)")
    p.add_argument("--no-bvh-compare", action="store_true",
                   help="skip the host SAH against device LBVH builder comparison")
    p.add_argument("--no-suns", action="store_true",
                   help="field config: skip the 256-sun time-to-SE comparison (and the "
                        "other configs)")
    p.add_argument("--no-others", action="store_true",
                   help="field config: skip the short runs of the other configs")
    p.add_argument("--cpu-seconds", type=float, default=10.0)
    p.add_argument("--ref-step-seconds", type=float, default=10.0)
    args = p.parse_args()
    if args.paths is None:
        args.paths = {"beamdown": 200_000_000, "mirror": 1_000_000}.get(args.config,
                                                                         100_000_000)
    if args.spp is None:
        args.spp = 16 if args.config == "pt" else 4
    if args.impl == "reference" and args.config in ("draft", "pt"):
        run_draw_reference(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.config in ("draft", "pt"):
        run_draw(args)
    elif args.config == "suns":
        run_suns(args)
    elif args.config == "adjoint":
        run_adjoint(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
