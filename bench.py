"""Benchmark of the render hot path: Stokes ray-samples/s of the full-Stokes polarized image
workload (256 x 256 screen over +-20 M, a = 0.5, theta_o = 60 deg, 1024 samples per ray, 64
thermal splats, 3 frequencies), one GPU per process.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--precision mixed|fp64]

One step = one render of every ray at every frequency (ks_render). `value` is device-resident
throughput (inputs and the FP64 plan/anchor table resident in HBM; the table, about 150 MB, is
larger than L2, so nothing is flushed between steps); `e2e` is the same metric through the public
Python API with host buffers (parameters uploaded, Stokes images read back every step). Under
torchrun every rank renders its own parameter set (weak scaling, no data-path collective) and the
step time is the max over ranks. `--impl reference` times the CPU oracle (the C++ FP64
restatement of the reference's path; the reference itself is Julia and cannot run here) on a
bounded sample of the same workload with every host thread.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Stokes ray-samples/s (full-Stokes polarized transport)"
UNIT = "ray-samples/s"

# Algorithmic FP32-pipe work per event of the polarized consumer and the march (flops: add, mul =
# 1, fma = 2, div = 1) and special-function-unit operations (sqrt, exp, log, sin, cos, atan, acos,
# pow count 1 each), counted from the kernel source (kerrsplat_b200/csrc/ks_march.cuh,
# ks_transfer.cuh, ks_lib.cu PolSink).
FLOPS = {"samples": 330, "valid_samples": 95, "splat_tests": 22, "weights": 32, "coefficients": 170,
         "frames": 115, "steps": 1150}
SFU = {"samples": 12, "valid_samples": 9, "splat_tests": 2, "weights": 1, "coefficients": 22, "frames": 4, "steps": 12}
# k_consume's DRAM traffic per ray-sample: ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch
# of this workload at full size (256x256, N = 1024, 3 frequencies: 2.1709e9 + 0.1235e9 B over 65536 x 1024
# ray-samples; reads = the FP32 sample stream, 32 B per ray-sample, partly still in L2 after k_stream
# writes it, + the plan; writes = segment states)
CONSUME_TRAFFIC_PER_RAY_SAMPLE = (2.170923e9 + 0.123528e9) / (65536 * 1024)


def rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(value, device=None):
    """The largest `value` over the ranks of the default process group (a step time, in ms)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            v = [x.strip() for x in l.split(",")]
            try:
                sm.append(float(v[0]))
                smax = float(v[1])
            except (ValueError, IndexError):
                continue
            for n, x in zip(names, v[3:7]):
                if x.lower() in ("active", "1"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def workload(seed_offset=0, res=256, nsamples=1024):
    from kerrsplat_b200 import scenes
    c = scenes.config2(res=res, N=nsamples)
    if seed_offset:
        rng = np.random.Generator(np.random.PCG64(1 + 1000 * seed_offset))
        c["params"] = scenes.thermal_params(rng, 64, c["a"])
    return c


def run_ours(args):
    import torch
    import torch.distributed as dist
    import kerrsplat_b200 as ks
    from kerrsplat_b200 import build
    rank, world, local = rank_info()
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    build.build(verbose=False)
    c = workload(seed_offset=rank, res=args.res, nsamples=args.nsamples)
    prec = {"mixed": ks.KS_MIXED, "mixed_geo64": ks.KS_MIXED_GEO64, "fp64": ks.KS_FP64}[args.precision]
    cache = ks.GeodesicCache(c["camera"], c["N"], device=local)
    ks.regenerate(cache, c["a"], c["theta_o"], marcher=ks.Fused(c["M"]))
    dev = torch.device("cuda", local)
    tuned = None
    if args.autotune and prec != ks.KS_FP64:
        tuned = ks.autotune(cache, ks.PolarizedSplats(c["params"]), [c["t_obs"]], c["nus"], c["L"], trials=1)
    model_dev = ks.PolarizedSplats(torch.tensor(c["params"], device=dev))
    times_dev = torch.tensor([c["t_obs"]], dtype=torch.float64, device=dev)
    nus_dev = torch.tensor(c["nus"], dtype=torch.float64, device=dev)
    nf = len(c["nus"])
    out_dev = torch.empty((nf, 1, cache.npix, 4), dtype=torch.float64, device=dev)
    units_per_step = cache.npix * c["N"] * 1 * nf
    stream = torch.cuda.ExternalStream(cache.stream(), device=dev)

    def step():
        ks.render(cache, model_dev, times_dev, nus_dev, c["L"], precision=prec, out=out_dev, order="sorted")

    for _ in range(args.warmup):
        step()
    # work-event counts of one render (the algorithmic-work model of the roofline)
    cache.count_events(True)
    step()
    counts = cache.event_counts()
    cache.count_events(False)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    cache.kernel_stats(reset=True)
    cache.consume_stats(reset=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
    ms_total = e0.elapsed_time(e1)
    render_ms, render_launches, all_launches = cache.kernel_stats(reset=True)
    consume_ms, consume_launches = cache.consume_stats(reset=True)
    ms_total = max_over_ranks(ms_total, dev)
    ms_step = ms_total / args.steps
    value = units_per_step * world / (ms_step / 1e3)

    # the same render captured as a CUDA graph (device-resident parameters; each replay rebuilds the
    # splat tables from them, marches, consumes, composes and unsorts): no host work per step
    graph = None
    try:
        if prec != ks.KS_MIXED:
            raise RuntimeError("the graph path captures the mixed render only")
        g = ks.capture_render(cache, model_dev, times_dev, nus_dev, c["L"], out=out_dev, order="sorted")
        for _ in range(2):
            g.replay(wait=False)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(args.steps):
            g.replay(wait=False)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        g.replay(wait=True)
        gms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dev)
        graph = {"ms_per_step": gms, "value": units_per_step * world / (gms / 1e3)}
        g.close()
    except Exception as exc:   # reported, not fatal: the headline is the ks_render path
        graph = {"error": str(exc)}

    # e2e: the public API with host buffers (parameters uploaded, images read back every step)
    model_host = ks.PolarizedSplats(c["params"])
    out_host = np.empty((nf, 1, cache.npix, 4))
    h2d = c["params"].nbytes + 8 * (1 + nf)
    d2h = out_host.nbytes
    ks.render(cache, model_host, [c["t_obs"]], c["nus"], c["L"], precision=prec, out=out_host)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    e2e_steps = max(1, min(args.steps, 5))
    for _ in range(e2e_steps):
        ks.render(cache, ks.PolarizedSplats(c["params"]), [c["t_obs"]], c["nus"], c["L"], precision=prec, out=out_host)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / e2e_steps
    e2e_ms = max_over_ranks(e2e_ms, dev)
    e2e_value = units_per_step * world / (e2e_ms / 1e3)

    # roofline of the dominant kernel: k_consume on the mixed path (the march runs before it in
    # k_stream, so its per-sample flops are left out), k_polarized<double> on the FP64 plain path;
    # algorithmic FP32 (FP64) work per launch / its CUDA-event time
    if prec != ks.KS_FP64 and consume_launches > 0:
        kname = "k_consume"
        flops = sum(FLOPS[k] * counts[k] for k in FLOPS if k != "samples")
        sfu = sum(SFU[k] * counts[k] for k in SFU if k != "samples")
        launch_ms = consume_ms / consume_launches
        launches_per_step = consume_launches / args.steps
        traffic = CONSUME_TRAFFIC_PER_RAY_SAMPLE * cache.npix * c["N"]
    else:
        kname = "k_polarized<double,1>"
        flops = sum(FLOPS[k] * counts[k] for k in FLOPS)
        sfu = sum(SFU[k] * counts[k] for k in SFU)
        launch_ms = render_ms / max(render_launches, 1)
        launches_per_step = render_launches / args.steps
        traffic = None
    flops_per_launch = flops / max(launches_per_step, 1)
    achieved = flops_per_launch / (launch_ms / 1e3) / 1e12
    pk = peaks()
    clocks = clk.summary()
    smax = pk.get("sm_max_mhz", 1965.0)
    fp32_peak = 148 * 128 * 2 * smax * 1e6 / 1e12   # nominal FP32 (non-tensor) FMA peak at max clock
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if prec == ks.KS_FP64 else "f32", "data": "synthetic (seeded PCG64 scene, cfg 2 distributions)",
        "config": {"workload": f"polarized image {args.res}x{args.res} +-20M, a=0.5, theta_o=60deg, N={args.nsamples}, M=64, 64 thermal splats, 86/230/345 GHz",
                   "precision": args.precision, "rays": cache.npix, "samples_per_ray": c["N"], "frequencies": nf,
                   "l2": "no flush: the per-ray FP64 plan + anchor table (~150 MB) exceeds the 126 MB L2"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                     "traffic": traffic, "traffic_source": "ncu DRAM bytes of one k_consume launch of this workload (256x256, N=1024, 3 frequencies)"
                     if traffic else None,
                     "peak_source": "nominal FP32 pipe (148 SMs x 128 lanes x 2 x max SM clock); MEASURED_PEAKS.json has no FP32 figure",
                     "kernel": kname, "kernel_ms": launch_ms, "flops_per_launch": flops_per_launch,
                     "sfu_ops_per_launch": sfu / max(launches_per_step, 1), "events": counts,
                     "hbm_frac": (traffic / (launch_ms / 1e3) / 1e9) / pk["hbm_gbs"] if traffic and pk.get("hbm_gbs") else None},
        "gpu_launches": int(all_launches),
        "graph": graph,
        "autotune": None if tuned is None else {"block": tuned[0], "units_per_warp": tuned[1], "ms": tuned[2]},
        "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(c, args.cpu_rays)
    if not args.no_gradient:
        line["chi2_grad"] = chi2_grad_bench(args, cache, c, dev, stream, world)
    if args.fp64_steps > 0 and prec != ks.KS_FP64:
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(args.fp64_steps):
            ks.render(cache, model_dev, times_dev, nus_dev, c["L"], precision=ks.KS_FP64, out=out_dev, order="sorted")
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms64 = e0.elapsed_time(e1) / args.fp64_steps
        line["fp64_plain"] = {"value": units_per_step / (ms64 / 1e3), "ms_per_step": ms64, "speedup_mixed_over_fp64": ms64 / ms_step}
    if rank == 0:
        print(json.dumps(line), flush=True)
    cache.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def chi2_grad_bench(args, cache, c, dev, stream, world):
    """chi^2 + gradient evaluations per second (configuration 3): the configuration-2 scene against a
    target rendered from parameters perturbed by 5% and 1% Gaussian pixel noise; one evaluation =
    forward + chi^2 + adjoint of all 64 x 21 parameters at the three frequencies. Mixed path timed on
    the device (data resident), end to end through the public API (host data and gradient), and the
    FP64 plain path (the reference's dual-sweep structure) once."""
    import torch
    import kerrsplat_b200 as ks
    from kerrsplat_b200 import scenes
    pt, rng = scenes.config3_target(c["params"])
    target = np.asarray(ks.render(cache, ks.PolarizedSplats(pt), [c["t_obs"]], c["nus"], c["L"], precision=ks.KS_MIXED))
    sigma = 0.01 * float(np.abs(target[..., 0]).max())
    data = target + sigma * rng.standard_normal(target.shape)
    model = ks.PolarizedSplats(torch.tensor(c["params"], device=dev))
    data_dev = torch.tensor(data, device=dev)
    grad_dev = torch.zeros(c["params"].size, dtype=torch.float64, device=dev)
    times, nus = [c["t_obs"]], c["nus"]

    def step(prec):
        return ks.chi2_gradient(cache, model, times, nus, c["L"], data_dev, sigma, precision=prec, dparams=grad_dev)

    for _ in range(max(1, args.warmup)):
        step(ks.KS_MIXED)
    steps = max(1, min(args.steps, 10))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record(stream)
    for _ in range(steps):
        chi2, _ = step(ks.KS_MIXED)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = max_over_ranks(e0.elapsed_time(e1) / steps, dev)
    # end to end: host parameters, host data, host gradient
    host_model = ks.PolarizedSplats(c["params"])
    t0 = time.perf_counter()
    for _ in range(steps):
        chi2_h, g_h = ks.chi2_gradient(cache, host_model, times, nus, c["L"], data, sigma, precision=ks.KS_MIXED)
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / steps, dev)
    out = {"metric": "chi^2+grad evals/s", "value": world * 1e3 / ms, "ms_per_eval": ms, "steps": steps,
           "workload": "config 3: config-2 scene (256x256, N=1024, 64 thermal splats, 86/230/345 GHz) vs a 5%-perturbed target + 1% noise",
           "parameters": int(c["params"].size), "chi2": float(chi2_h),
           "e2e": {"value": world * 1e3 / e2e_ms, "ms_per_eval": e2e_ms, "h2d_bytes_per_step": int(data.nbytes + c["params"].nbytes),
                   "d2h_bytes_per_step": int(c["params"].nbytes + 8)}}
    # the same evaluation captured as a CUDA graph (device-resident model and data) and replayed
    try:
        cg = ks.capture_chi2_gradient(cache, model, times, nus, c["L"], data_dev, sigma)
        cg.replay()
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(steps):
            cg.replay(wait=False)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        cg.replay(wait=True)
        gms = max_over_ranks(e0.elapsed_time(e1) / steps, dev)
        out["graph"] = {"value": world * 1e3 / gms, "ms_per_eval": gms, "chi2": float(cg.chi2.item())}
        cg.close()
    except Exception as exc:   # reported, not fatal
        out["graph"] = {"error": str(exc)}
    if args.fp64_steps > 0:
        step(ks.KS_FP64)   # stored samples are built on the first FP64 call after a regenerate
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(args.fp64_steps):
            step(ks.KS_FP64)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms64 = e0.elapsed_time(e1) / args.fp64_steps
        g64 = ks.chi2_gradient(cache, host_model, times, nus, c["L"], data, sigma, precision=ks.KS_FP64)[1]
        rel = float(np.linalg.norm(np.asarray(g_h) - np.asarray(g64)) / np.linalg.norm(g64))
        out["fp64_plain"] = {"value": 1e3 / ms64, "ms_per_eval": ms64, "speedup_mixed_over_fp64": ms64 / ms,
                             "grad_rel_l2_mixed_vs_fp64": rel}
    return out


def run_movie(args):
    """The batched movie (configuration 4): 32 frames x 4 frequencies of a 512 x 512 screen, a = 0.94,
    theta_o = 163 deg, slow light, uneven samples per ray (128 to 2048 by Mino time), 256 splats (85
    thermal on trajectory knots, 85 power-law, 86 kappa), all frames and frequencies in one mixed
    render. One step = the whole movie; the metric counts every ray's own samples."""
    import torch
    import kerrsplat_b200 as ks
    from kerrsplat_b200 import build, scenes
    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    build.build(verbose=False)
    c = scenes.config4(res=args.res, nframes=args.frames)
    cache = ks.GeodesicCache(c["camera"], c["N"], device=local)
    ks.regenerate(cache, c["a"], c["theta_o"], uneven=(c["density"], c["nmin"]))
    nsamp = cache.nsamples_per_ray
    model = ks.CompositeModel(ks.KnotSplats(c["thermal"], c["knots"], c["knot_times"]), ks.PowerLawSplats(c["powerlaw"]),
                              ks.KappaSplats(c["kappa"]))
    dev = torch.device("cuda", local)
    nf, nt = len(c["nus"]), len(c["times"])
    out = torch.empty((nf, nt, cache.npix, 4), dtype=torch.float64, device=dev)
    stream = torch.cuda.ExternalStream(cache.stream(), device=dev)
    units = float(nsamp.sum()) * nf * nt
    for _ in range(args.warmup):
        ks.render(cache, model, c["times"], c["nus"], c["L"], precision=ks.KS_MIXED, out=out, order="sorted")
    # work-event counts of one movie (the consumer's samples, splat tests, weights, evaluations, steps)
    cache.count_events(True)
    ks.render(cache, model, c["times"], c["nus"], c["L"], precision=ks.KS_MIXED, out=out, order="sorted")
    events = cache.event_counts()
    cache.count_events(False)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(args.steps):
            ks.render(cache, model, c["times"], c["nus"], c["L"], precision=ks.KS_MIXED, out=out, order="sorted")
        e1.record(stream)
        torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / args.steps
    finite = bool(torch.isfinite(out).all())
    line = {"metric": "Stokes ray-samples/s (batched movie)", "value": units / (ms / 1e3), "unit": "ray-samples/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded PCG64 scene, cfg 4 distributions)",
            "config": {"workload": f"batched movie {args.res}x{args.res} +-15M, a=0.94, theta_o=163deg, {nt} frames x 4 freqs, uneven N "
                                   f"(mean {nsamp.mean():.0f}, {nsamp.min()}-{nsamp.max()}), 85 knot + 85 power-law + 86 kappa splats",
                       "ray_samples_per_step": units, "finite": finite, "events": events},
            "clocks": {k: clk.summary()[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")}}
    if args.fp64_steps > 0:
        # the FP64 plain path on the first frame only (one march per frame and frequency)
        sub = units / nt
        torch.cuda.synchronize(dev)
        e0.record(stream)
        ks.render(cache, model, c["times"][:1], c["nus"], c["L"], precision=ks.KS_FP64, out=out[:, :1].contiguous(), order="sorted")
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms64 = e0.elapsed_time(e1)
        line["fp64_plain"] = {"value": sub / (ms64 / 1e3), "ms_first_frame": ms64, "speedup_mixed_over_fp64": (sub / (ms64 / 1e3)) and
                              (units / (ms / 1e3)) / (sub / (ms64 / 1e3))}
    print(json.dumps(line), flush=True)
    cache.close()


def run_fit(args):
    """The minibatched fit iteration (configuration 5): for each of the 16 parameter sets, the forward
    image, the 3xTF32 DFT onto 2000 baselines, chi^2 against its noisy target, the adjoint DFT and the
    reverse pass (ks_vis_chi2_gradient), and the Gauss-Newton normal-equation product along the
    gradient, g^T J^T J g = |J g|^2 (one J v pass and one DFT): the curvature of the matrix-free
    normal equations. One step = all sets; the FP64 plain path is timed on one set."""
    import torch
    import kerrsplat_b200 as ks
    from kerrsplat_b200 import build, scenes
    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    build.build(verbose=False)
    c = scenes.config5(res=args.res, N=args.nsamples, nsets=args.sets)
    cache = ks.GeodesicCache(c["camera"], c["N"], device=local)
    ks.regenerate(cache, c["a"], c["theta_o"])
    rng = c["rng"]
    targets = []
    for p in c["sets"]:
        pt = p + 0.05 * np.maximum(np.abs(p), 0.1) * rng.standard_normal(p.shape)
        img = np.asarray(ks.render(cache, ks.PolarizedSplats(pt), [c["t_obs"]], [c["nu"]], c["L"], precision=ks.KS_MIXED))[0, 0]
        V = np.asarray(ks.visibilities(cache, img, c["u"], c["v"], c["psize"], c["scale"], precision=ks.KS_MIXED))
        sig = np.maximum(0.02 * np.abs(V), 1e-3 * np.abs(V).max())
        noise = sig * (rng.standard_normal(V.shape) + 1j * rng.standard_normal(V.shape)) / np.sqrt(2)
        targets.append((V + noise, sig))

    def one_set(q, prec, times=None):
        p, (vis, sig) = c["sets"][q], targets[q]
        m = ks.PolarizedSplats(p)
        t0 = time.perf_counter()
        chi2, g = ks.vis_chi2_gradient(cache, m, c["t_obs"], c["nu"], c["L"], c["u"], c["v"], vis, sig, c["psize"], c["scale"], precision=prec)
        t1 = time.perf_counter()
        jv = ks.jvp(cache, m, [c["t_obs"]], [c["nu"]], c["L"], g, precision=prec)[0, 0, 0]
        t2 = time.perf_counter()
        Vd = np.asarray(ks.visibilities(cache, jv, c["u"], c["v"], c["psize"], c["scale"], precision=prec))
        curv = float(np.sum(np.abs(Vd / sig) ** 2))
        if times is not None:
            times.update({"chi2_grad_ms": (t1 - t0) * 1e3, "jvp_ms": (t2 - t1) * 1e3, "dft_ms": (time.perf_counter() - t2) * 1e3})
        return chi2, float(np.sum(g * g)), curv

    for _ in range(args.warmup):
        one_set(0, ks.KS_MIXED)
    torch.cuda.synchronize()
    per_set = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for q in range(len(c["sets"])):
            t1 = time.perf_counter()
            tm = {}
            chi2, gg, curv = one_set(q, ks.KS_MIXED, tm)
            per_set.append(dict({"splats": int(c["counts"][q]), "ms": (time.perf_counter() - t1) * 1e3, "chi2": chi2,
                                 "gn_step": -0.5 * gg / max(curv, 1e-300)}, **tm))
    ms_iter = (time.perf_counter() - t0) * 1e3 / args.steps
    line = {"metric": "fit iterations/s (minibatched)", "value": 1e3 / ms_iter, "unit": "iterations/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_iter, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded PCG64 scene, cfg 5 distributions)",
            "config": {"workload": f"minibatched fit {args.res}x{args.res} +-16M, a=0.7, theta_o=30deg, N={c['N']}, 230 GHz, "
                                   f"{len(c['sets'])} thermal sets of {int(c['counts'].min())}-{int(c['counts'].max())} splats, "
                                   f"{len(c['u'])} baselines, 3xTF32 DFT",
                       "iteration": "per set: forward + DFT + chi^2 + adjoint DFT + reverse pass + J g + DFT (GN curvature g^T J^T J g)",
                       "timing": "wall clock around the synchronous calls (host data)"},
            "per_set": per_set[:len(c["sets"])]}
    if args.fp64_steps > 0:
        t1 = time.perf_counter()
        tm = {}
        one_set(0, ks.KS_FP64, tm)
        ms64 = (time.perf_counter() - t1) * 1e3
        line["fp64_plain"] = dict({"set": 0, "splats": int(c["counts"][0]), "ms": ms64, "speedup_mixed_over_fp64": ms64 / per_set[0]["ms"]}, **tm)
    print(json.dumps(line), flush=True)
    cache.close()


def run_dft(args):
    """The visibility transform of configuration 5 (a 1024 x 1024 four-Stokes image onto 2000 baselines,
    and the adjoint seed back), mixed precision: per step one ks_visibilities and one ks_vis_seed call
    from host arrays (the e2e figure: host->device copies of the image and weights, device->host copies
    of V and the seed, inside the timed region), with the L2 flushed between steps (a 256 MB write).
    The two 3xTF32 GEMMs of a step (4096 x 4000 x 1024 and 1024 x 4096 x 4000) are timed with CUDA
    events (ks_gemm_stats) on the tcgen05 kernel and on the mma.sync fallback; the FP64 direct sums
    (the reference's algorithm) are timed once."""
    import torch
    import kerrsplat_b200 as ks
    from kerrsplat_b200 import build, scenes
    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    build.build(verbose=False)
    c = scenes.config5(res=args.res, N=8, nsets=1)
    cache = ks.GeodesicCache(c["camera"], 8, device=local)
    ks.regenerate(cache, c["a"], c["theta_o"])
    rng = np.random.Generator(np.random.PCG64(11 + rank))
    npix = c["camera"].npix
    img = np.abs(rng.standard_normal((npix, 4))) * np.array([1.0, 0.2, 0.2, 0.05])
    nuv = len(c["u"])
    w = rng.standard_normal((nuv, 4)) + 1j * rng.standard_normal((nuv, 4))
    # pinned host buffers for the image and the seed (the two large copies of a step)
    img_h = torch.from_numpy(img).pin_memory().numpy()
    seed_h = torch.empty((npix, 4), dtype=torch.float64).pin_memory().numpy()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def step():
        V = ks.visibilities(cache, img_h, c["u"], c["v"], c["psize"], c["scale"], precision=ks.KS_MIXED)
        S = ks.vis_seed(cache, w, c["u"], c["v"], c["psize"], c["scale"], precision=ks.KS_MIXED, out=seed_h)
        return V, S

    res = {}
    for path in ("mma.sync", "tcgen05"):
        cache.set_tensor_path(path)
        for _ in range(args.warmup):
            step()
        cache.gemm_stats(reset=True)
        tot = 0.0
        clocks = ClockSampler(local)
        with clocks:
            for _ in range(args.steps):
                flush.fill_(1)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                V, S = step()
                tot += time.perf_counter() - t0
        gms, gl, gfl = cache.gemm_stats(reset=True)
        res[path] = {"ms_per_step": tot * 1e3 / args.steps, "gemm_ms_per_step": gms / args.steps, "gemm_launches": gl,
                     "gemm_tflops": gfl / (gms * 1e-3) / 1e12, "V": V, "S": S.copy(), "clocks": clocks.summary()}
    cache.set_tensor_path("tcgen05")
    t0 = time.perf_counter()
    V64 = ks.visibilities(cache, img_h, c["u"], c["v"], c["psize"], c["scale"], precision=ks.KS_FP64)
    S64 = ks.vis_seed(cache, w, c["u"], c["v"], c["psize"], c["scale"], precision=ks.KS_FP64)
    ms64 = (time.perf_counter() - t0) * 1e3
    rel = lambda x, y: float(np.linalg.norm(x - y) / np.linalg.norm(y))
    tc, ms = res["tcgen05"], res["mma.sync"]
    pk = peaks()
    tf32_peak = pk["bf16_tflops"] / 2 if "bf16_tflops" in pk else 1590.0 / 2
    h2d = img.nbytes + w.nbytes + 2 * 8 * nuv * 2
    d2h = 8 * nuv * 8 + npix * 4 * 8
    line = {"metric": "visibility transforms/s (forward + adjoint)", "value": 1e3 / tc["ms_per_step"], "unit": "transforms/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tc["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (3xTF32)", "data": "synthetic (seeded image, cfg 5 baselines)",
            "config": {"workload": f"config-5 DFT: {args.res}x{args.res} x 4 Stokes image onto {nuv} baselines and the adjoint seed back",
                       "gemms": f"T = A Tu^T ({4 * args.res} x {2 * nuv} x {args.res}), S = Tu C^T ({args.res} x {4 * args.res} x {2 * nuv})",
                       "l2": "flushed between steps (256 MB write); each GEMM reads the operands its producer kernels just wrote",
                       "timing": "wall clock around the host-array calls (e2e); CUDA events around each GEMM"},
            "e2e": {"value": 1e3 / tc["ms_per_step"], "unit": "transforms/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "tensor", "achieved": tc["gemm_tflops"], "peak": tf32_peak, "unit": "TFLOP/s",
                         "frac": tc["gemm_tflops"] / tf32_peak, "traffic": None, "kernel": "k_gemm_tc",
                         "kernel_ms_per_step": tc["gemm_ms_per_step"],
                         "peak_source": "TF32 dense = half the measured BF16 burst (MEASURED_PEAKS.json bf16_tflops)"
                         if "bf16_tflops" in pk else "TF32 dense = half the fallback BF16 burst",
                         "flops": "3 x 2 M N K per GEMM (the three TF32 products are issued)"},
            "mma_sync": {"ms_per_step": ms["ms_per_step"], "gemm_ms_per_step": ms["gemm_ms_per_step"], "gemm_tflops": ms["gemm_tflops"],
                         "V_rel_vs_tcgen05": rel(ms["V"], tc["V"]), "seed_rel_vs_tcgen05": rel(ms["S"], tc["S"])},
            "fp64_direct": {"ms": ms64, "V_rel_mixed_vs_fp64": rel(tc["V"], V64), "seed_rel_mixed_vs_fp64": rel(tc["S"], S64),
                            "speedup_mixed_over_fp64": ms64 / tc["ms_per_step"]},
            "clocks": tc["clocks"]}
    print(json.dumps(line), flush=True)
    cache.close()


def run_shards(args):
    """Configuration 3's chi^2 + gradient with the rays sharded over ranks (kerrsplat_b200.shard): each
    rank regenerates and evaluates its own rays, then one all-reduce of [chi^2, dparams] (1345 FP64).
    Under torchrun every rank evaluates its shard and the step time (evaluation + all-reduce) is the
    max over ranks. On one process the shards of 2, 4 and 8 ranks run one after another on this GPU:
    each shard's evaluation is timed with CUDA events (data already on the device), and the largest
    one against the whole screen's time / ranks is the load balance of that partition; the sums of
    the shards' chi^2 and gradients are checked against the whole screen's."""
    import torch
    import kerrsplat_b200 as ks
    from kerrsplat_b200 import build, scenes
    from kerrsplat_b200.shard import RayShard, allreduce_sum
    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    build.build(verbose=False)
    c = scenes.config2(res=args.res, N=args.nsamples)
    cache = ks.GeodesicCache(c["camera"], c["N"], device=local)
    ks.regenerate(cache, c["a"], c["theta_o"])
    pt, rng = scenes.config3_target(c["params"])
    target = np.asarray(ks.render(cache, ks.PolarizedSplats(pt), [c["t_obs"]], c["nus"], c["L"], precision=ks.KS_MIXED))
    sigma = 0.01 * float(np.abs(target[..., 0]).max())
    data = torch.tensor(target + sigma * rng.standard_normal(target.shape), device=dev)
    model = ks.PolarizedSplats(torch.tensor(c["params"], device=dev))
    times, nus = [c["t_obs"]], c["nus"]
    steps = max(1, min(args.steps, 10))
    nparam = c["params"].size

    def timed(sh_cache, d):
        # the timed calls add into one buffer; the checked gradient comes from a call on a zeroed one
        # (buffers written on torch's stream are waited for before the library's stream reads them)
        acc = torch.zeros(nparam, dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        for _ in range(max(1, args.warmup)):
            ks.chi2_gradient(sh_cache, model, times, nus, c["L"], d, sigma, precision=ks.KS_MIXED, dparams=acc)
        stream = torch.cuda.ExternalStream(sh_cache.stream(), device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(steps):
            ks.chi2_gradient(sh_cache, model, times, nus, c["L"], d, sigma, precision=ks.KS_MIXED, dparams=acc)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        grad = torch.zeros(nparam, dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        chi2, _ = ks.chi2_gradient(sh_cache, model, times, nus, c["L"], d, sigma, precision=ks.KS_MIXED, dparams=grad)
        return e0.elapsed_time(e1) / steps, chi2, grad.cpu().numpy()

    full_ms, full_chi2, full_g = timed(cache, data)
    line = {"metric": "chi^2+grad evals/s (rays sharded over ranks)", "unit": "evals/s", "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded PCG64 scene, cfg 3 target)",
            "config": {"workload": f"config 3: {args.res}x{args.res}, N={args.nsamples}, 64 thermal splats, 86/230/345 GHz, 1344 parameters",
                       "l2": "no flush: the per-ray plan + anchor table exceeds the 126 MB L2 at 256x256"}}
    if world > 1:
        import torch.distributed as dist
        sh = RayShard(c["camera"], c["N"], c["a"], c["theta_o"], rank=rank, world=world, device=local)
        d = sh.take(data, 2)
        if sh.cache is None:
            raise RuntimeError("empty shard")
        g = torch.zeros(1 + nparam, dtype=torch.float64, device=dev)

        def step():
            # [chi^2, dparams] of this rank's rays, then the sum over ranks (the library's call returns
            # after its stream finishes; the all-reduce follows on torch's stream)
            g.zero_()
            torch.cuda.current_stream(dev).synchronize()
            chi2, _ = ks.chi2_gradient(sh.cache, model, times, nus, c["L"], d, sigma, precision=ks.KS_MIXED, dparams=g[1:])
            g[0] = chi2
            dist.all_reduce(g, op=dist.ReduceOp.SUM)
        for _ in range(max(1, args.warmup)):
            step()
        dist.barrier()
        torch.cuda.synchronize(dev)
        stream = torch.cuda.current_stream(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        dist.barrier()
        ms = max_over_ranks(e0.elapsed_time(e1) / steps, dev)
        gv = g.cpu().numpy()
        line.update({"value": 1e3 / ms, "ms_per_step": ms, "whole_screen_one_gpu_ms": full_ms,
                     "chi2_rel_vs_one_gpu": abs(gv[0] - full_chi2) / full_chi2,
                     "grad_rel_vs_one_gpu": float(np.linalg.norm(gv[1:] - full_g) / np.linalg.norm(full_g))})
        sh.close()
        if rank == 0:
            print(json.dumps(line), flush=True)
        dist.barrier()
        dist.destroy_process_group()
        cache.close()
        return
    emulated = {}
    for w in (2, 4, 8):
        for layout in ("contiguous", "strided"):
            per, chi2s, gsum = [], 0.0, np.zeros_like(full_g)
            for r in range(w):
                sh = RayShard(c["camera"], c["N"], c["a"], c["theta_o"], rank=r, world=w, layout=layout, device=local)
                ms_r, chi2_r, g_r = timed(sh.cache, sh.take(data, 2))
                per.append(ms_r)
                chi2s += chi2_r
                gsum += g_r
                sh.close()
            vec = allreduce_sum(np.concatenate([[chi2s], gsum]))   # one process: the identity
            emulated[f"{w}/{layout}"] = {"shard_ms": [round(x, 3) for x in per], "max_shard_ms": max(per),
                                         "balance": max(per) / (full_ms / w), "sum_shard_ms": sum(per),
                                         "chi2_rel": abs(vec[0] - full_chi2) / full_chi2,
                                         "grad_rel": float(np.linalg.norm(vec[1:] - full_g) / np.linalg.norm(full_g))}
    line.update({"value": 1e3 / full_ms, "ms_per_step": full_ms,
                 "emulated_ranks": emulated,
                 "note": "one GPU: each rank's shard timed alone, one after another; balance = the largest shard's time / "
                         "(whole screen's time / ranks); a rank's step adds one all-reduce of 1345 FP64 values"})
    print(json.dumps(line), flush=True)
    cache.close()


def cpu_sample(c, nrays, seed=7):
    rng = np.random.Generator(np.random.PCG64(seed))
    idx = np.sort(rng.choice(c["camera"].npix, size=min(nrays, c["camera"].npix), replace=False))
    return idx


def cpu_baseline(c, nrays):
    """The CPU oracle (C++ FP64 restatement, OpenMP over rays, every host thread) on a bounded
    random sample of the workload's rays at all frequencies."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    oracle.set_threads(os.cpu_count() or 1)
    idx = cpu_sample(c, nrays)
    cam = c["camera"]
    t0 = time.perf_counter()
    for nu in c["nus"]:
        oracle.polarized_image(c["a"], c["theta_o"], cam.alpha[idx], cam.beta[idx], c["N"], c["M"], [("thermal", c["params"], None)],
                               c["t_obs"], nu, c["L"])
    dt = time.perf_counter() - t0
    units = idx.size * c["N"] * len(c["nus"])
    return {"value": units / dt, "unit": UNIT, "cores": oracle.num_threads(), "kind": "port",
            "sample": f"{idx.size} random rays of the 256x256 workload x {c['N']} samples x {len(c['nus'])} frequencies ({dt:.1f} s)",
            "seconds": dt, "units": units, "rays": int(idx.size)}


def run_reference(args):
    rank, world, local = rank_info()
    if rank != 0:
        return
    c = workload()
    units, secs = 0, 0.0
    for k in range(args.warmup + args.steps):
        b = cpu_baseline(c, args.cpu_rays)
        if k >= args.warmup:
            units += b["units"]
            secs += b["seconds"]
    v = units / secs
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": secs / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded PCG64 scene, cfg 2 distributions)",
            "config": {"workload": f"{b['rays']} seeded random rays of the polarized image 256x256 +-20M, a=0.5, theta_o=60deg, N=1024, M=64, "
                                   "64 thermal splats, 86/230/345 GHz",
                       "note": "one step renders the ray sample at every frequency; ms_per_step is that sample's time"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": b["cores"], "kind": "port", "sample": b["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "mixed_geo64", "fp64"])
    ap.add_argument("--cpu-rays", type=int, default=1024)
    ap.add_argument("--fp64-steps", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-gradient", action="store_true", help="skip the chi^2 + gradient measurement")
    ap.add_argument("--autotune", action=argparse.BooleanOptionalAction, default=True,
                    help="time the consumer's launch shapes before the timed steps (ks_autotune)")
    ap.add_argument("--res", type=int, default=None, help="screen resolution (default: the workload's; smaller cases for profiling)")
    ap.add_argument("--nsamples", type=int, default=None, help="samples per ray (default: the workload's)")
    ap.add_argument("--workload", default="polarized", choices=["polarized", "movie", "fit", "dft", "shards"],
                    help="polarized: configurations 2 and 3 (the headline); movie: configuration 4; fit: configuration 5; "
                         "dft: configuration 5's visibility transform on both tensor-core kernels; "
                         "shards: configuration 3's chi^2 + gradient with the rays sharded over ranks")
    ap.add_argument("--sets", type=int, default=16, help="fit: parameter sets")
    ap.add_argument("--frames", type=int, default=32, help="movie frames")
    args = ap.parse_args()
    # the sizes of each workload's configuration unless given
    dres, dn = {"polarized": (256, 1024), "movie": (512, 2048), "fit": (1024, 512), "dft": (1024, 8),
                "shards": (256, 1024)}[args.workload]
    args.res = dres if args.res is None else args.res
    args.nsamples = dn if args.nsamples is None else args.nsamples
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "movie":
        run_movie(args)
    elif args.workload == "fit":
        run_fit(args)
    elif args.workload == "dft":
        run_dft(args)
    elif args.workload == "shards":
        run_shards(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
