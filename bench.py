"""Benchmark: surface points/s of batched AR surface generation on B200.

Workload (default ``batched``): 256 independent surfaces in one call, as the
batched-realisations configuration specifies -- t uniform in [64, 512]; x and
y drawn log-uniformly from {32, 64, 128, 256}; AR order per surface from
{4, 6, 8, 10}^3; standing or propagating ACF with b in [0.03, 0.1]
(standing: a=1.5, c=0.8, d=0.5; propagating: a=1, c=0.6, d=0.3, e=0.2);
surface i uses dcmt parameter set i mod 16 and seed 42 + i.  Synthetic
inputs, all drawn from numpy's generator seeded with 42 (per rank: 42 + 1000 *
rank).  A step is one call of the batched generator: white noise for every
surface, the FP32 compensated AR filter over all surfaces in one persistent
launch, and the variance renormalisation.  Coefficients are fitted once
(FP64) before timing, as model set-up.

`value` is whole-job points/s with buffers resident in HBM; `e2e` is the same
call writing into pinned host buffers (device->host copies inside the timed
region).  The plain FP64 path (the reference's exact summation order, one
surface after another) is timed on the same batch and reported beside it.
The CPU baseline is the oracle's restatement of the reference's OpenMP block
wavefront on a bounded sample of the batch.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
    python bench.py --stage velocity|ar|ar64|batch|nit|ma [...]   (one stage alone)
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "surface points/s: batched FP32 vs plain FP64 AR on 1 B200; p50/p99 latency"


def _load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


PEAKS = _load_peaks()
N_SURFACES = 256
MT_SETS = 16


# --------------------------------------------------------------------- workload
def make_batch(rank: int = 0, n: int = N_SURFACES):
    rng = np.random.default_rng(42 + 1000 * rank)
    sizes = [32, 64, 128, 256]
    orders = [4, 6, 8, 10]
    out = []
    for i in range(n):
        nt = int(rng.integers(64, 513))
        nx = int(sizes[rng.integers(0, 4)])
        ny = int(sizes[rng.integers(0, 4)])
        order = tuple(int(orders[rng.integers(0, 4)]) for _ in range(3))
        kind = "propagating" if rng.random() < 0.5 else "standing"
        b = float(rng.uniform(0.03, 0.1))
        out.append(dict(shape=(nt, nx, ny), order=order, kind=kind, b=b,
                        seed=42 + i + 1000 * rank, mtset=i % MT_SETS))
    return out


def acf_params(s):
    if s["kind"] == "standing":
        return dict(kind=0, amplitude=1.5, velocity=0.8, alpha=[s["b"]] * 3, beta=[0.5, 0.5])
    return dict(kind=1, amplitude=1.0, velocity=0.6, alpha=[s["b"]] * 3, beta=[0.3, 0.2])


def fit_batch(batch):
    import arma_b200 as A
    for s in batch:
        p = acf_params(s)
        phi, var = A.ar_fit_analytic(p["kind"], s["order"], p["amplitude"], p["velocity"],
                                     p["alpha"], p["beta"])
        s["phi"], s["var"], s["acf0"] = phi, var, p["amplitude"]
    return batch


def mt_sets():
    """The 16 dcmt parameter sets of period 2^19937 - 1 (arma_b200/data/mt.dat,
    created by ``python -m arma_b200.dcmt -n 16 -p 19937 -s 42``)."""
    import arma_b200 as A
    path = os.path.join(ROOT, "arma_b200", "data", "mt.dat")
    n = A.mt_file_count(path)
    if n != MT_SETS:
        raise RuntimeError(f"{path}: {n} parameter sets, the workload needs {MT_SETS}")
    return [A.mt_file_read(path, k) for k in range(n)]


def points(batch):
    return int(sum(np.prod(s["shape"]) for s in batch))


def flops(batch):
    """Algorithmic AR work: 2 (P - 1) flops per point."""
    return float(sum(np.prod(s["shape"]) * 2 * (np.prod(s["order"]) - 1) for s in batch))


def shard_value(points_per_rank: int, steps: int, elapsed_s: float, world: int) -> float:
    """Whole-job points/s of a weakly scaled run: every rank processes its own
    batch of `points_per_rank` points per step; `elapsed_s` is the max over
    ranks of the timed region."""
    return world * points_per_rank * steps / elapsed_s


def reduce_max(x: float, device: str) -> float:
    """Max of x over the ranks of the default process group (x itself when
    there is none)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# --------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------- CPU arms
def cpu_sample(batch, seconds_hint: float):
    """A bounded sample of the batch with the batch's work mix, about
    `seconds_hint` of CPU work: surfaces are visited in a seeded random order
    and each is taken while the sample's flops stay within the budget, so the
    sample's point-weighted order matches the batch's (reported beside it)."""
    rate = 1.5e9  # flop/s per core, rough planning figure for the scalar loop
    cores = os.cpu_count() or 1
    budget = seconds_hint * rate * cores
    order = np.random.default_rng(7).permutation(len(batch))
    chosen, acc = [], 0.0
    for k in order:
        s = batch[int(k)]
        f = np.prod(s["shape"]) * 2 * (np.prod(s["order"]) - 1)
        if acc + f <= budget:
            chosen.append(s)
            acc += f
    if not chosen:
        chosen = [min(batch, key=lambda s: np.prod(s["shape"]) * np.prod(s["order"]))]
    return chosen


def weighted_taps(batch):
    """Point-weighted mean number of AR coefficients P of a set of surfaces."""
    return flops(batch) / (2.0 * points(batch)) + 1.0


def run_cpu(sample, sets, nthreads):
    """Reference CPU path (oracle restatement of the OpenMP backend): white noise
    per partition from per-thread MTs, block wavefront filter, renormalisation."""
    import oracle as O
    nthreads = nthreads or (os.cpu_count() or 1)
    ps = [O.MtParams.from_buffer_copy(sets[k % len(sets)]) for k in range(nthreads)]
    t0 = time.perf_counter()
    for s in sample:
        z = O.ar_generate_omp(s["shape"], s["phi"], float(np.sqrt(s["var"])), ps,
                              [s["seed"] + k for k in range(nthreads)], nthreads)
        O.variance_renorm(z, s["acf0"])
    return time.perf_counter() - t0


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    batch = fit_batch(make_batch(0))
    sets = mt_sets()
    sample = cpu_sample(batch, 8.0)
    cores = os.cpu_count() or 1
    for _ in range(args.warmup):
        run_cpu(sample[:1], sets, cores)
    times = [run_cpu(sample, sets, cores) for _ in range(args.steps)]
    pts = points(sample)
    t = max(statistics.median(times), 1e-9)
    v = pts / t
    desc = (f"{len(sample)} of the {N_SURFACES} surfaces in seeded random order ({pts} points, "
            f"point-weighted P {weighted_taps(sample):.0f} against {weighted_taps(batch):.0f} for "
            f"the whole batch); OpenMP block wavefront with per-thread MT noise + "
            f"renormalisation, {cores} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "points/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "batched-256-surfaces", "sample": desc},
        "flops_per_s": flops(sample) / t,
        "cpu_baseline": {"value": v, "unit": "points/s", "cores": cores, "kind": "port",
                         "sample": desc, "flops_per_s": flops(sample) / t},
        "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# --------------------------------------------------------------------- GPU arm
def gpu_arm(args):
    import torch
    import torch.distributed as dist

    import arma_b200 as A
    from arma_b200 import capi

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    batch = fit_batch(make_batch(rank)[:args.surfaces or N_SURFACES])
    sets = mt_sets()
    ctx = A.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)  # events below bracket the library's stream
    bufs32 = [torch.empty(s["shape"], dtype=torch.float32, device="cuda") for s in batch]
    surf32 = [capi.make_surface(s["shape"], s["phi"], s["var"], s["acf0"],
                                sets[s["mtset"] % len(sets)], s["seed"], b.data_ptr())
              for s, b in zip(batch, bufs32)]
    npts = points(batch)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return reduce_max(x, "cuda")

    # ---- device-resident FP32 compensated batch, with the speed settings the
    # autotuner picks for this batch (result-invariant; tuning time untimed)
    tuned_dev, tune_dev_ms = ctx.autotune(surf32, A.FP32C)
    for _ in range(args.warmup):
        ctx.batch_generate(surf32, A.FP32C)
    barrier()
    ctx.set_profiling(True)
    ctx.profile_reset()
    launches0 = ctx.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        ev0.record(stream)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            ctx.batch_generate(surf32, A.FP32C)
        ctx.synchronize()
        ev1.record(stream)
        barrier()
        wall = time.perf_counter() - t0
    launches = ctx.launch_count() - launches0
    elapsed = max(ev0.elapsed_time(ev1) / 1e3, 1e-9)
    elapsed = max_over_ranks(elapsed)
    ar_ms, ar_n = ctx.profile("ar32c")
    prof = {k: ctx.profile(k) for k in ("mt", "noise", "ar32c", "renorm")}
    ctx.set_profiling(False)
    value = shard_value(npts, args.steps, elapsed, world)

    # ---- e2e: same call into pinned host buffers
    e2e = None
    tuned_host = None
    if args.skip_e2e:
        host = []
    else:
        host = [torch.empty(s["shape"], dtype=torch.float32, pin_memory=True) for s in batch]
        surfh = [capi.make_surface(s["shape"], s["phi"], s["var"], s["acf0"],
                                   sets[s["mtset"] % len(sets)], s["seed"], h.data_ptr())
                 for s, h in zip(batch, host)]
        tuned_host, tune_host_ms = ctx.autotune(surfh, A.FP32C, host=True)
        ctx.batch_generate(surfh, A.FP32C, host=True)
        barrier()
        h2d0, d2h0 = ctx.transfer_bytes()
        t0 = time.perf_counter()
        e2e_steps = args.steps
        for _ in range(e2e_steps):
            ctx.batch_generate(surfh, A.FP32C, host=True)
        barrier()
        e2e_t = max_over_ranks(time.perf_counter() - t0)
        h2d1, d2h1 = ctx.transfer_bytes()
        e2e = world * npts * e2e_steps / e2e_t
        e2e_h2d = (h2d1 - h2d0) // e2e_steps
        e2e_d2h = (d2h1 - d2h0) // e2e_steps
        # parity spot check of the host copy against the device result
        assert torch.equal(host[0], bufs32[0].cpu())
        # the device->host link of this box: plain pinned copies of about
        # 1 GB of the same surfaces, best of three, CUDA events on one stream
        pick, nb = [], 0
        for k in range(len(batch)):
            pick.append(k)
            nb += host[k].numel() * 4
            if nb >= 1 << 30:
                break
        link = 0.0
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for k in pick:
                host[k].copy_(bufs32[k], non_blocking=True)
            e1.record()
            e1.synchronize()
            link = max(link, nb / (e0.elapsed_time(e1) * 1e-3) / 1e9)
        e2e_link = {"d2h_link_gbs": link,
                    "copy_bound_ms": e2e_d2h / (link * 1e9) * 1e3,
                    "ms_per_call": e2e_t / e2e_steps * 1e3}
        ctx.set_tuning(tuned_dev)  # the device-resident legs below
    del bufs32

    # ---- plain FP64 path on the same batch (surface after surface)
    plain = None
    if not args.skip_plain:
        bufs64 = [torch.empty(s["shape"], dtype=torch.float64, device="cuda") for s in batch]
        surf64 = [capi.make_surface(s["shape"], s["phi"], s["var"], s["acf0"],
                                    sets[s["mtset"] % len(sets)], s["seed"], b.data_ptr())
                  for s, b in zip(batch, bufs64)]
        ctx.batch_generate(surf64, A.FP64)  # builds and caches the plane graphs
        barrier()
        t0 = time.perf_counter()
        ctx.batch_generate(surf64, A.FP64)
        barrier()
        t64 = max_over_ranks(time.perf_counter() - t0)
        plain = world * npts / t64
        del bufs64

    # ---- roofline of the dominant kernel (ar32c)
    peaks = PEAKS
    sm_max = float(peaks.get("sm_max_mhz", 1965.0))
    fp32_peak = 148 * 128 * 2 * sm_max * 1e6 / 1e12  # TFLOP/s at the max SM clock
    per_launch_flops = flops(batch)  # one ar32c pass over the batch per step
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "ar32c_dram_traffic.json")) as f:
            tr = json.load(f)
        traffic = (tr["dram_bytes_read"] + tr["dram_bytes_write"]) * npts / tr["points"]
    except (OSError, KeyError, ValueError):
        pass
    ar_s = ar_ms / 1e3 / max(args.steps, 1)
    achieved = per_launch_flops / ar_s / 1e12 if ar_s > 0 else None

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        sample = cpu_sample(batch, args.cpu_seconds / 2)
        cores = os.cpu_count() or 1
        t = run_cpu(sample, sets, cores)
        cpu = {"value": points(sample) / t, "unit": "points/s", "cores": cores, "kind": "port",
               "flops_per_s": flops(sample) / t,
               "sample": f"{len(sample)} surfaces of the batch in seeded random order "
                         f"({points(sample)} points, point-weighted P {weighted_taps(sample):.0f} "
                         f"against {weighted_taps(batch):.0f} for the batch), OpenMP block "
                         f"wavefront restatement, {t:.1f} s"}

    full = None
    if not args.skip_full:
        full = full_path(A, capi, ctx, batch, sets, 2, stream)
        full["value"] *= world  # every rank runs its own batch
        full["ratio_over_plain_fp64_ar"] = (full["value"] / plain) if plain else None
    prec = None
    if rank == 0 and not args.skip_precision:
        prec = precision_report(A, capi, ctx)

    serving = None
    if world == 1 and not args.skip_serve:
        serving = serve_bench(A, args.serve_seconds)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True,
            "flops_per_s": flops(batch) * world * args.steps / elapsed,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (compensated), f64 fit",
            "data": "synthetic (seeded numpy draws; no external dataset)",
            "config": {"workload": "batched-256-surfaces",
                       "surfaces": len(batch), "points_per_rank": npts,
                       "orders": "{4,6,8,10}^3", "precision": "fp32c",
                       "l2": "inputs larger than L2 (%.1f GB per rank)" % (npts * 4 / 1e9),
                       "parallelism": f"dp{world} (independent surfaces per rank)"},
            "e2e": {"value": e2e, "unit": "points/s", "h2d_bytes_per_step": e2e_h2d,
                    "d2h_bytes_per_step": e2e_d2h, "steps": e2e_steps, **e2e_link,
                    "copies": "counted by the library (arma_ctx_transfer_bytes): host->device "
                              "task lists, parameter sets and coefficient tables; device->host "
                              "surfaces, scales and accepted-pair counts"} if e2e else None,
            "plain_fp64": {"value": plain, "unit": "points/s",
                           "ratio_fp32c_over_fp64": (value / plain) if plain else None},
            "gpu_launches": launches,
            "tuning": {"device": tuned_dev.as_dict(),
                       "host_output": tuned_host.as_dict() if tuned_host else None,
                       "how": "arma_autotune on this batch before timing: coordinate descent "
                              "over the MT segment length, the filter's CTAs per SM and the "
                              "host-output group split; results are bit-identical across "
                              "settings"},
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in prof.items()},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak,
                         "unit": "TFLOP/s", "frac": (achieved / fp32_peak) if achieved else None,
                         "traffic": traffic,
                         "traffic_unit": "bytes per launch (ncu dram read+write, 24-surface "
                                         "capture scaled by points)",
                         "algorithmic_bytes": npts * 8,
                         "note": "ar32c: 2(P-1) flop per point over the batch / ar32c device "
                                 "time; peak = 148 SMs x 128 FP32 lanes x 2 x max SM clock "
                                 "(MEASURED_PEAKS.json has no FP32 figure)"},
            "cpu_baseline": cpu,
            "full_path": full,
            "precision_fp32c_vs_fp64": prec,
            "latency": ({"p50_ms": serving["p50_ms_at_50pct"], "p99_ms": serving["p99_ms_at_50pct"],
                         "p99_128x128x64_ms": serving["p99_128x128x64_ms_at_50pct"],
                         "load": 0.5, "source": "serving"} if serving else None),
            "serving": serving,
            "clocks": clk.summary(),
            "wall_s_timed": wall,
        }
        print(json.dumps(line))
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


# --------------------------------------------------------------------- full path
def full_path(A, capi, ctx, batch, sets, steps, stream):
    """The batched FP32 compensated path end to end on the device: noise, AR
    filter, renormalisation and the skew-normal NIT (skewness 0.3: alpha
    1.499; 1024-node inverse-CDF table applied in the renormalisation's scale
    pass) for every surface in one call, then the linear velocity potential at
    z = 0 on every slice of every surface (infinite depth), batched by slice
    shape.  Returns points/s and the per-stage device milliseconds of one
    step."""
    import torch
    order = sorted(range(len(batch)), key=lambda k: batch[k]["acf0"])
    total = points(batch)
    flat = torch.empty(total, dtype=torch.float32, device="cuda")
    vel = torch.empty(total, dtype=torch.float32, device="cuda")
    surfs, groups, off = [], {}, 0
    for k in order:
        s = batch[k]
        n = int(np.prod(s["shape"]))
        surfs.append(capi.make_surface(s["shape"], s["phi"], s["var"], s["acf0"],
                                       sets[s["mtset"] % len(sets)], s["seed"],
                                       flat[off:].data_ptr()))
        nt, nx, ny = s["shape"]
        groups.setdefault((nx, ny), []).append(
            (flat[off:].data_ptr(), vel[off:].data_ptr(), nt, list(range(nt)), 1.0))
        off += n
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]

    # the NIT table applied in the renormalisation's scale pass
    tables = [A.nit_table(A.NIT_SKEW_NORMAL, [0.0, 1.0, 1.499], float(np.sqrt(batch[k]["acf0"])),
                          1024, 5.0) for k in order]

    def step(record):
        if record:
            ev[0].record(stream)
        ctx.batch_generate_nit(surfs, A.FP32C, tables)
        if record:
            ev[1].record(stream)
        for (nx, ny), jobs in groups.items():
            ctx.velocity_linear_batch(jobs, nx, ny, A.FP32C, float("inf"), [0.0])
        if record:
            ev[2].record(stream)

    step(False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    stage = np.zeros(2)
    for _ in range(steps):
        step(True)
        torch.cuda.synchronize()
        stage += [ev[i].elapsed_time(ev[i + 1]) for i in range(2)]
    wall = time.perf_counter() - t0
    dev_ms = float(stage.sum()) / steps
    # velocity roofline, algorithmic work per slice of N = nx ny points at nz
    # depths: 5 N log2 N flop per complex FFT (one forward, nz inverse) + 6 N nz
    # for the window product; N 4 bytes read and nz N 4 bytes written (FP32)
    nz, vflop, vbytes = 1, 0.0, 0.0
    for (nx, ny), jobs in groups.items():
        n = nx * ny
        nslices = sum(j[2] for j in jobs)
        vflop += nslices * (5.0 * n * np.log2(n) * (1 + nz) + 6.0 * n * nz)
        vbytes += nslices * 4.0 * n * (1 + nz)
    vel_s = stage[1] / steps / 1e3
    sm_max = float(PEAKS.get("sm_max_mhz", 1965.0))
    fp32_peak = 148 * 128 * 2 * sm_max * 1e6 / 1e12
    hbm_peak = float(PEAKS.get("hbm_gbs", 6650.0))
    v_tf = vflop / vel_s / 1e12
    v_gb = vbytes / vel_s / 1e9
    vroof = {"flop_per_step": vflop, "bytes_per_step": vbytes,
             "fp32": {"achieved": v_tf, "peak": fp32_peak, "unit": "TFLOP/s",
                      "frac": v_tf / fp32_peak},
             "hbm": {"achieved": v_gb, "peak": hbm_peak, "unit": "GB/s", "frac": v_gb / hbm_peak},
             "binding": "fp32" if v_tf / fp32_peak > v_gb / hbm_peak else "hbm",
             "note": "all velocity kernels (zeta_t, FFTs, window, factor_waves) over the "
                     "algorithmic FFT + window work; peaks as the ar32c roofline (FP32 at the "
                     "max SM clock) and MEASURED_PEAKS.json's copy bandwidth"}
    return {"value": total / (dev_ms / 1e3), "unit": "points/s", "steps": steps,
            "velocity_roofline": vroof,
            "ms_per_step": dev_ms, "wall_ms_per_step": wall / steps * 1e3,
            "stage_ms": {"noise_ar_renorm_nit": stage[0] / steps,
                         "velocity_z0": stage[1] / steps},
            "workload": "batched-256-surfaces + skew-normal NIT (LUT 1024 nodes) + velocity "
                        "potential at z=0 on every slice (infinite depth)"}


def precision_report(A, capi, ctx):
    """FP32 compensated against FP64 on the 400 x 128 x 128 propagating model
    of order 10^3 (zeta, variance, ACF, velocity at z in {0,-1,-2,-4}) and the
    NIT moments of the 512 x 256 x 256 model (first 64 slices)."""
    import torch
    from arma_b200.precision import compare_surfaces, field_error
    phi, var = A.ar_fit_analytic(A.ACF_PROPAGATING, (10, 10, 10), 1.0, 0.6, [0.04] * 3, [0.3, 0.2])
    mt = A.mt19937_params()

    def pair(shape):
        z64 = torch.empty(shape, dtype=torch.float64, device="cuda")
        z32 = torch.empty(shape, dtype=torch.float32, device="cuda")
        for z, prec in ((z64, A.FP64), (z32, A.FP32C)):
            ctx.batch_generate([capi.make_surface(shape, phi, var, 1.0, mt, 42, z.data_ptr())], prec)
        ctx.synchronize()
        return z64, z32

    z64, z32 = pair((400, 128, 128))
    out = {"zeta_400x128x128": compare_surfaces(z64, z32)}
    zs = [0.0, -1.0, -2.0, -4.0]
    v64 = torch.empty((400, 4, 128, 128), dtype=torch.float64, device="cuda")
    v32 = torch.empty((400, 4, 128, 128), dtype=torch.float32, device="cuda")
    for z, v, prec in ((z64, v64, A.FP64), (z32, v32, A.FP32C)):
        ctx.velocity_linear(z.data_ptr(), z.shape, prec, (1.0, 1.0, 1.0), float("inf"), zs,
                            list(range(400)), v.data_ptr())
    ctx.synchronize()
    ve = field_error(v64, v32)
    # a slice whose wave-number range (a discontinuous function of the
    # surface) resolves differently on the FP32 surface stands out by far
    per_slice = (v32.double() - v64).abs().amax(dim=(1, 2, 3))
    over = per_slice > 2e-4 * ve["max_ref"]
    ve["slices_over_2e-4_of_max"] = int(over.sum())
    ve["max_abs_other_slices"] = float(per_slice[~over].max()) if bool((~over).any()) else None
    out["velocity_400x128x128_z4"] = ve
    del z64, z32, v64, v32
    z64, z32 = pair((512, 256, 256))
    w64, w32 = z64[:64].contiguous(), z32[:64].contiguous()
    del z64, z32
    ctx.nit_apply(A.NIT_SKEW_NORMAL, [0.0, 1.0, 1.499], 1.0, A.NIT_BISECTION, w64.numel(), A.FP64,
                  w64.data_ptr(), interval=(-10.0, 10.0), eps=1e-10, max_iter=100)
    ctx.nit_apply(A.NIT_SKEW_NORMAL, [0.0, 1.0, 1.499], 1.0, A.NIT_LUT, w32.numel(), A.FP32C,
                  w32.data_ptr(), lut_nodes=1024, lut_range=5.0)
    ctx.synchronize()
    out["nit_skew_normal_512x256x256_first64"] = compare_surfaces(w64, w32)
    return out


# --------------------------------------------------------------------- serving
SERVE_SIDES = (64, 128, 256)
SERVE_T = 64


def serve_bench(A, seconds_per_load: float, seed: int = 42):
    """Serving workload: streams of x = y in {64, 128, 256}, AR order 8^3
    (standing / propagating ACFs alternating), FP32 filter with the velocity
    potential at z = 0, chunks of 64 slices delivered into pinned host memory.
    Capacity is measured closed-loop (four chunks queued for each of 48
    streams); then Poisson arrivals at 10-90 % of it, each a request for the
    next chunk of a random stream or, with probability 0.1, a new stream that
    replaces a random one of the same size.  Latency = submit -> chunk and
    velocity in host memory (the server's clock)."""
    import torch
    rng = np.random.default_rng(seed)
    mt = A.mt19937_params()
    fits = [A.ar_fit_analytic(A.ACF_STANDING, (8, 8, 8), 1.5, 0.8, [0.05] * 3, [0.5, 0.5]),
            A.ar_fit_analytic(A.ACF_PROPAGATING, (8, 8, 8), 1.0, 0.6, [0.04] * 3, [0.3, 0.2])]
    srv = A.Server(chunk_slices=SERVE_T, velocity=1, z_levels=[0.0], max_inflight=3)
    next_seed = [1000]

    def open_stream(k, side):
        phi, var = fits[k % 2]
        next_seed[0] += 1
        return srv.open_stream(side, side, phi, var, 1.0, mt, next_seed[0])

    streams = [(open_stream(k, SERVE_SIDES[k % 3]), SERVE_SIDES[k % 3]) for k in range(48)]
    pool = {side: [(torch.empty((SERVE_T, side, side), dtype=torch.float32).pin_memory(),
                    torch.empty((SERVE_T, 1, side, side), dtype=torch.float32).pin_memory())
                   for _ in range(68)] for side in SERVE_SIDES}
    inflight = {}

    def submit(i):
        sid, side = streams[i]
        b = pool[side].pop()
        inflight[srv.submit(sid, b[0].data_ptr(), b[1].data_ptr())] = (b, side)

    def collect(done):
        for d in done:
            b, side = inflight.pop(d["request"])
            pool[side].append(b)
            if d["status"] != 0:
                raise RuntimeError(f"serving request failed: {d} {srv.last_failure()}")
            d["side"] = side
        return done

    try:
        for _ in range(2):  # warm-up: every stream's first chunks, scratch growth
            for i in range(len(streams)):
                submit(i)
            collect(srv.wait(len(streams), 120000))
        zero = {}
        for i in range(3):
            lat = []
            for _ in range(15):
                submit(i)
                lat.append(collect(srv.wait(1))[0]["latency_ms"])
            zero[f"{streams[i][1]}x{streams[i][1]}x{SERVE_T}"] = float(np.median(lat))
        npts = 0
        t0 = time.perf_counter()
        for _ in range(4):
            for i in range(len(streams)):
                submit(i)
                npts += SERVE_T * streams[i][1] ** 2
        collect(srv.wait(4 * len(streams), 120000))
        dt = time.perf_counter() - t0
        cap = 4 * len(streams) / dt
        loads = []
        for load in (0.1, 0.3, 0.5, 0.7, 0.9):
            lam = load * cap
            n = max(50, int(lam * seconds_per_load))
            arrivals = np.cumsum(rng.exponential(1.0 / lam, n))
            picks = rng.integers(0, len(streams), n)
            fresh = rng.random(n) < 0.1
            res = []
            start = time.perf_counter()
            for a, i, new in zip(arrivals, picks, fresh):
                while time.perf_counter() - start < a:
                    res += collect(srv.poll(256, 0))
                while not pool[streams[i][1]]:
                    res += collect(srv.poll(256, 1))
                if new:
                    side = streams[i][1]
                    srv.close_stream(streams[i][0])
                    streams[i] = (open_stream(int(i), side), side)
                submit(i)
            res += collect(srv.wait(n - len(res), 120000))
            span = time.perf_counter() - start
            lat = np.array([r["latency_ms"] for r in res])
            l128 = np.array([r["latency_ms"] for r in res if r["side"] == 128])
            loads.append({"load": load, "rate_per_s": lam, "requests": n,
                          "achieved_per_s": n / span,
                          "p50_ms": float(np.percentile(lat, 50)),
                          "p99_ms": float(np.percentile(lat, 99)),
                          "p50_128_ms": float(np.percentile(l128, 50)) if l128.size else None,
                          "p99_128_ms": float(np.percentile(l128, 99)) if l128.size else None,
                          "mean_batch": float(np.mean([r["batch_size"] for r in res]))})
        st = srv.stats()
    finally:
        srv.close()
    half = next(x for x in loads if x["load"] == 0.5)
    return {
        "workload": "serving: 48 streams x,y in {64,128,256}, order 8^3, chunks of 64 slices, "
                    "fp32c + velocity at z=0, outputs to pinned host memory, Poisson arrivals, "
                    "10% new streams",
        "capacity_chunks_per_s": cap, "capacity_points_per_s": npts / dt,
        "zero_load_p50_ms": zero, "loads": loads,
        "p50_ms_at_50pct": half["p50_ms"], "p99_ms_at_50pct": half["p99_ms"],
        "p99_128x128x64_ms_at_50pct": half["p99_128_ms"],
        "server": {k: st[k] for k in ("batches", "completed", "redone", "launches")},
    }


# --------------------------------------------------------------------- stages
def _timed(ctx, stream, fn, warm=3, reps=5):
    """Device milliseconds per call of fn (CUDA events on the library's
    stream, `warm` untimed calls first)."""
    import torch
    for _ in range(warm):
        fn()
    ctx.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def run_stage(args):
    """One stage of the path in isolation, for timing and for ncu captures of
    its kernels (``--stage NAME``); prints one line with the device time.

    velocity  linear velocity solver on every slice of one propagating-wave
              surface (order 10^3, FP32 compensated) of slices x side x side,
              nz depth levels in {0, -1, -2, -4, ...}, infinite depth
    ar        batched FP32 path (MT, noise, AR filter, renormalisation) on
              `surfaces` standing-wave surfaces of one shape and order
    ar64      the plain FP64 path on the same
    batch     the bench batch's first `surfaces` surfaces, FP32 compensated
    full      the bench's full path (noise + AR + renormalisation, NIT table,
              velocity at z = 0 on every slice) on the first `surfaces`
    nit       skew-normal NIT (1024-node table over +-5 sigma, or the per-point
              bisection with --bisection) in place over one surface
    ma        MA filter (zeta = eps - theta * eps) of one surface, random
              coefficients of the given order"""
    import torch
    import arma_b200 as A
    from arma_b200 import capi
    ctx = A.Context(0)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    shape = (args.slices, args.side, args.side)
    pts = int(np.prod(shape))
    tag = "fp64" if args.fp64 else "fp32"
    if args.stage == "velocity":
        phi, var = A.ar_fit_analytic(A.ACF_PROPAGATING, (10, 10, 10), 1.0, 0.6, [0.04] * 3,
                                     [0.3, 0.2])
        prec, dt = (A.FP64, torch.float64) if args.fp64 else (A.FP32C, torch.float32)
        z = torch.empty(shape, dtype=dt, device="cuda")
        ctx.batch_generate([capi.make_surface(shape, phi, var, 1.0, A.mt19937_params(), 42,
                                              z.data_ptr())], prec)
        zs = [0.0, -1.0, -2.0, -4.0, -8.0, -16.0, -32.0, -64.0][:args.nz]
        out = torch.empty((args.slices, args.nz, args.side, args.side), dtype=dt, device="cuda")
        tidx = list(range(args.slices))
        ms = _timed(ctx, stream, lambda: ctx.velocity_linear(
            z.data_ptr(), shape, prec, (1.0, 1.0, 1.0), float("inf"), zs, tidx, out.data_ptr()))
        print(f"velocity {args.slices}x{args.side}x{args.side} nz={args.nz} {tag}: "
              f"{ms:.3f} ms/call, {pts / ms / 1e6:.2f} G points/s")
    elif args.stage in ("ar", "ar64"):
        order = (args.order,) * 3
        phi, var = A.ar_fit_analytic(A.ACF_STANDING, order, 1.5, 0.8, [0.05] * 3, [0.5, 0.5])
        prec, dt = (A.FP64, torch.float64) if args.stage == "ar64" else (A.FP32C, torch.float32)
        nsurf = args.surfaces or 8
        bufs = [torch.empty(shape, dtype=dt, device="cuda") for _ in range(nsurf)]
        surfs = [capi.make_surface(shape, phi, var, 1.5, A.mt19937_params(), 42 + k, b.data_ptr())
                 for k, b in enumerate(bufs)]
        ms = _timed(ctx, stream, lambda: ctx.batch_generate(surfs, prec),
                    warm=1 if args.stage == "ar64" else 3, reps=1 if args.stage == "ar64" else 5)
        n = nsurf * pts
        flop = n * 2.0 * (np.prod(order) - 1)
        print(f"{args.stage} {nsurf} x {shape} order {order}: {ms:.3f} ms/call, "
              f"{n / ms / 1e6:.2f} G points/s, {flop / ms / 1e9:.2f} TFLOP/s algorithmic")
    elif args.stage == "batch":
        batch = fit_batch(make_batch(0)[:args.surfaces or N_SURFACES])
        sets = mt_sets()
        bufs = [torch.empty(b["shape"], dtype=torch.float32, device="cuda") for b in batch]
        surfs = [capi.make_surface(b["shape"], b["phi"], b["var"], b["acf0"],
                                   sets[b["mtset"] % len(sets)], b["seed"], z.data_ptr())
                 for b, z in zip(batch, bufs)]
        ms = _timed(ctx, stream, lambda: ctx.batch_generate(surfs, A.FP32C))
        print(f"batch {len(batch)} surfaces ({points(batch)} points): {ms:.3f} ms/call, "
              f"{points(batch) / ms / 1e6:.2f} G points/s")
    elif args.stage == "full":
        batch = fit_batch(make_batch(0)[:args.surfaces or N_SURFACES])
        r = full_path(A, capi, ctx, batch, mt_sets(), 2, stream)
        ctx.set_profiling(True)
        ctx.profile_reset()
        full_path(A, capi, ctx, batch, mt_sets(), 1, stream)
        kern = {k: round(ctx.profile(k)[0] / 2, 3) for k in ("mt", "noise", "ar32c", "renorm")}
        ctx.set_profiling(False)
        print(f"full {len(batch)} surfaces ({points(batch)} points): {r['ms_per_step']:.2f} ms/step "
              f"{json.dumps(r['stage_ms'])} kernels (ms per step, profiled) {json.dumps(kern)} "
              f"velocity roofline {json.dumps(r['velocity_roofline'])}")
    elif args.stage == "nit":
        z = torch.randn(shape, dtype=torch.float32, device="cuda")
        method = A.NIT_BISECTION if args.bisection else A.NIT_LUT
        ms = _timed(ctx, stream, lambda: ctx.nit_apply(
            A.NIT_SKEW_NORMAL, [0.0, 1.0, 1.499], 1.0, method, pts, A.FP32C, z.data_ptr(),
            interval=(-10.0, 10.0), eps=1e-6, max_iter=100, lut_nodes=1024, lut_range=5.0))
        print(f"nit {'bisection' if args.bisection else 'lut'} {shape}: {ms:.3f} ms/call, "
              f"{pts * 8 / ms / 1e6:.1f} GB/s of 8 B per point")
    elif args.stage == "ma":
        order = tuple(int(v) for v in args.ma_order.split(","))
        rng = np.random.default_rng(1)
        theta = rng.normal(0.0, 0.2 / np.sqrt(np.prod(order)), order)
        prec, dt = (A.FP64, torch.float64) if args.fp64 else (A.FP32C, torch.float32)
        eps = torch.randn(shape, dtype=dt, device="cuda")
        z = torch.empty_like(eps)
        ms = _timed(ctx, stream, lambda: ctx.ma_filter(theta, shape, prec, eps.data_ptr(),
                                                         z.data_ptr()))
        flop = pts * 2.0 * int(np.prod(order))
        print(f"ma {shape} order {order} {tag}: {ms:.3f} ms/call, {pts / ms / 1e6:.2f} G points/s, "
              f"{flop / ms / 1e9:.2f} TFLOP/s algorithmic")
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--skip-plain", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--surfaces", type=int, default=None,
                    help="use the first N surfaces of the batch (profiling runs)")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-serve", action="store_true")
    ap.add_argument("--skip-full", action="store_true")
    ap.add_argument("--skip-precision", action="store_true")
    ap.add_argument("--serve-seconds", type=float, default=1.5,
                    help="Poisson phase length per load level")
    ap.add_argument("--stage", choices=["velocity", "ar", "ar64", "batch", "full", "nit", "ma"],
                    help="time one stage in isolation (profiling runs); see run_stage")
    ap.add_argument("--side", type=int, default=128)
    ap.add_argument("--slices", type=int, default=400)
    ap.add_argument("--nz", type=int, default=4)
    ap.add_argument("--order", type=int, default=8)
    ap.add_argument("--ma-order", default="20,10,10")
    ap.add_argument("--fp64", action="store_true")
    ap.add_argument("--bisection", action="store_true")
    args = ap.parse_args()
    if args.stage:
        run_stage(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
