#!/usr/bin/env python
"""Benchmark of the physical-optics Shack-Hartmann WFS frame.

Workload (default): NFIRAOS-like LGS, 30 m telescope with 3.6 m obstruction,
6 LGS WFS at 35" radius, 60x60 subapertures of 0.5 m (2820 valid), 16x16 OPD
points, 32x32 FFT, 6x6 pixels of 1", 7 von Karman layers on 2048^2 FP32
screens (synthetic, seeded), Gaussian sodium layer at 90 km (10 km FWHM) from
an LLT 8 m off axis, 500 photons/subaperture with 3 e- read noise, matched
filter gradients.  One step = one frame of all 6 WFS: ray trace, uplink OTF,
imaging, noise, gradients.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

The b200 arm prints one JSON line with the device-timed throughput (value),
the end-to-end throughput through the C ABI with host results (e2e), the
roofline of the dominant kernel and the reference's own CPU path timed on
this host (cpu_baseline).  The reference arm times the reference's own C for
the path (oracle/_ref, all host threads) on the same workload.  Under
torchrun each rank runs an independent replica (no collective on the data
path); the job value is the units of all ranks over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thr = threading.Thread(target=self._read, daemon=True)
            self.thr.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init():
    from maos_b200 import replicas
    return replicas.init("nccl")


def allreduce_max(x: float, ws: int, device) -> float:
    from maos_b200 import replicas
    return replicas.max_over_ranks(x, ws, device)


def barrier(ws: int, device):
    from maos_b200 import replicas
    replicas.barrier(ws, device)


# ---------------------------------------------------------------------------
def algorithmic_traffic(cfg, nsa, npix, nopd, notf, nwfs, nlayer):
    """Algorithmic bytes per launch of the two main kernels (minimum traffic)."""
    ints = (nsa * notf * notf * 8 if cfg.get("has_llt") else notf * notf * 4)  # ETF (shared) or nominal
    ints += nsa * nopd * nopd * 4                                             # amplitude (shared)
    ints += nwfs * nsa * nopd * nopd * 4                                      # OPD of every WFS
    ints += nwfs * nsa * npix * (4 + 8)                                       # ints out + matched filter
    ints += nwfs * (nsa * 4 + nsa * 8)                                        # i0sum + gradients
    ray = nwfs * nsa * nopd * nopd * (nlayer * 4 + 4)                         # all WFS in one launch
    return ints, ray


def fft_flops_per_image(notf):
    """Nominal FFT flop count per subaperture image: three 2-D transforms."""
    n2 = notf * notf
    return 3 * 5 * n2 * math.log2(n2)


def tc_mma_flops_per_image():
    """BF16 MMA flops the tensor-core imaging kernel executes per subaperture
    image: per 4-image tile, 2a/2b/4a 6 MMAs and 4b 12 MMAs of 128x64x16, 6a 12
    of 128x32x16 and 6b 12 of 128x16x16 (three split terms, zero padding included)."""
    tile = 30 * 128 * 64 * 16 * 2 + 12 * 128 * 32 * 16 * 2 + 12 * 128 * 16 * 16 * 2
    return tile / 4


def cpu_baseline(cfg, wl_layers, screens, seconds=15.0, max_frames=40):
    from oracle import ref
    ncpu = os.cpu_count() or 1
    r = ref.RefPowfs(cfg, nthread=ncpu)
    ref.atm_set(screens, wl_layers)
    dt = cfg.get("dt", 1.0 / 800)
    ref.frame_full_mt(r, 0, 0, dt)  # warm plans and caches
    t = 0.0
    n = 0
    while t < seconds and n < max_frames:
        _, _, dt_s = ref.frame_full_mt(r, n % cfg["nwfs"], n + 1, dt, seed=n + 1, noisy=True)
        t += dt_s
        n += 1
    return {"value": r.nsa * n / t, "unit": "subap-images/s", "cores": ncpu, "kind": "reference",
            "sample": f"{n} single-WFS frames of {cfg['name']} ({r.nsa} subapertures each): 7-layer ray trace, "
                      f"LLT uplink, wfsints, addnoise, matched filter; reference C (oracle/_ref), FFT stand-in "
                      f"for FFTW, NTHREAD={ncpu}"}


def run_reference(args, cfg):
    ws, rank, local = dist_init()
    if rank != 0:
        return 0
    from oracle import ref
    from maos_b200.setup import screens as mkscreens
    from maos_b200.workload import wind
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmaosref.so is not built"}))
        return 0
    ncpu = os.cpu_count() or 1
    r = ref.RefPowfs(cfg, nthread=ncpu)
    a = cfg["atm"]
    n = a["nx"]
    scr = mkscreens(n, n, a["dx"], a["r0"], a["L0"], a["wt"], 1)
    vx, vy = wind(cfg, 1)
    o = -n / 2 * a["dx"]
    layers = [dict(nx=n, ny=n, dx=a["dx"], ox=o, oy=o, ht=float(h), vx=float(vx[i]), vy=float(vy[i]))
              for i, h in enumerate(a["ht"])]
    ref.atm_set(scr, layers)
    dt = cfg.get("dt", 1.0 / 800)
    for i in range(args.warmup):
        ref.frame_full_mt(r, i % cfg["nwfs"], i, dt, seed=i + 1)
    times = []
    for k in range(args.steps):
        _, _, t = ref.frame_full_mt(r, k % cfg["nwfs"], args.warmup + k, dt, seed=k + 7)
        times.append(t)
    tot = sum(times)
    value = r.nsa * args.steps / tot
    line = {
        "impl": "reference", "metric": "subaperture images/s", "value": value, "unit": "subap-images/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": cfg["name"], "step": "one single-WFS frame (reference CPU path)"},
        "cpu_baseline": {"value": value, "unit": "subap-images/s", "cores": ncpu, "kind": "reference",
                         "sample": f"{args.steps} single-WFS frames of {cfg['name']} ({r.nsa} subapertures)"},
        "e2e": {"value": value, "unit": "subap-images/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_b200(args, cfg):
    import torch
    from maos_b200 import shwfs
    from maos_b200.workload import build
    ws, rank, local = dist_init()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    form = shwfs.SHWFS_FORM_TC if args.form == "tc" else shwfs.SHWFS_FORM_FFT
    wl = build(cfg, device=local, seed=1 + rank, noisy=True, form=form)
    ctx = wl.ctx
    nwfs = len(wl.wfs)
    units_per_step = nwfs * wl.nsa
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    variant = ctx.autotune(wl.wfs[0], wl.wfs[-1] + 1, nrep=5)
    isim = 0
    for _ in range(args.warmup):
        wl.frame(isim)
        isim += 1
    ctx.sync()
    barrier(ws, dev)
    clk = ClockSampler(local)
    clk.start()
    time.sleep(0.5)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with torch.cuda.stream(ext):
        for k in range(args.steps):
            flush.zero_()  # L2 flush between timed steps (not timed)
            starts[k].record(ext)
            wl.frame(isim)
            ends[k].record(ext)
            isim += 1
    ctx.sync()
    torch.cuda.synchronize(dev)
    clocks = clk.stop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    tot_ms = allreduce_max(sum(step_ms), ws, dev)
    barrier(ws, dev)
    value = units_per_step * args.steps * ws / (tot_ms * 1e-3)

    # stage timing of the same frames (profiled pass, separate from the timed one)
    ctx.profile_enable(True)
    nprof = min(args.steps, 20)
    with torch.cuda.stream(ext):
        for k in range(nprof):
            flush.zero_()
            wl.frame(isim)
            isim += 1
    ctx.sync()
    stages = ctx.profile_read()
    ctx.profile_enable(False)
    launches_per_step = sum(n for _, n in stages.values()) / nprof

    # end to end through the C ABI: queue + sync with host gradients each step,
    # into one host buffer the loop owns (as a C caller passes its own)
    ctx.copy_counters()
    gbuf = np.empty(sum(2 * ctx.wfs_nsa[i] for i in wl.wfs))
    e2e_s = 0.0
    for k in range(args.steps):
        with torch.cuda.stream(ext):
            flush.zero_()
        ctx.sync()
        t0 = time.perf_counter()
        wl.frame(isim)
        wl.frame_sync(out=gbuf)
        e2e_s += time.perf_counter() - t0
        isim += 1
    h2d, d2h = ctx.copy_counters()
    e2e_s = allreduce_max(e2e_s, ws, dev)
    e2e = units_per_step * args.steps * ws / e2e_s

    # roofline of the dominant kernel
    hbm, bf16, src = _peaks()
    nlayer = len(cfg["atm"]["ht"])
    ints_bytes, ray_bytes = algorithmic_traffic(cfg, wl.nsa, wl.npix, wl.setup.nopd, wl.setup.notf, nwfs, nlayer)
    st = {k: dict(ms_per_launch=(ms / n if n else 0.0), launches_per_step=n / nprof, ms_per_step=ms / nprof)
          for k, (ms, n) in stages.items()}
    ints_ms = st["ints"]["ms_per_launch"]
    ray_ms = st["raytrace"]["ms_per_step"]  # the WFS pupils, plus any LLT pupils traced in a second launch
    ints_gbs = ints_bytes / (ints_ms * 1e-3) / 1e9 if ints_ms else 0.0
    ray_gbs = ray_bytes / (ray_ms * 1e-3) / 1e9 if ray_ms else 0.0
    flops = fft_flops_per_image(wl.setup.notf) * units_per_step
    fp32_peak = 148 * 128 * 2 * 1.965e9 / 1e12  # nominal FP32 CUDA-core peak, TFLOP/s
    ints_tf = flops / (ints_ms * 1e-3) / 1e12 if ints_ms else 0.0
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get(f"{cfg['name']}:{args.form}:ints")
    src_note = f"{src} (MEASURED_PEAKS.json)" if src == "measured" else "fallback"
    raytrace = {"kernel": "geom_kernel", "achieved": ray_gbs, "peak": hbm, "unit": "GB/s", "frac": ray_gbs / hbm,
                "algorithmic_bytes_per_launch": ray_bytes}
    if args.form == "tc":
        tflops = units_per_step * tc_mma_flops_per_image() / (ints_ms * 1e-3) / 1e12 if ints_ms else 0.0
        post_ms = st["post"]["ms_per_launch"]
        roofline = {"kernel": "ints_tc_kernel (tcgen05 BF16x3 DFT imaging)", "bound": "tensor",
                    "achieved": tflops, "peak": bf16, "unit": "TFLOP/s", "frac": tflops / bf16,
                    "peak_source": src_note + " bf16_tflops, burst", "traffic": traffic,
                    "flops_per_launch": units_per_step * tc_mma_flops_per_image(),
                    "hbm": {"achieved": ints_gbs, "peak": hbm, "unit": "GB/s", "frac": ints_gbs / hbm,
                            "algorithmic_bytes_per_launch": ints_bytes},
                    "post": {"kernel": "noise_grad_kernel", "ms_per_launch": post_ms},
                    "raytrace": raytrace}
    else:
        if wl.setup.notf == 64:
            kname = "ints_n64_kernel (fused imaging, noise, gradients; half-spectrum transforms)"
            knote = ("the kernel moves its algorithmic bytes at this rate but is bound by shared-memory traffic "
                     "and issue (ncu: issue active 66 %, L1/shared 73 %, HBM 3 %); compute gives its FFT flop rate")
        else:
            kname = "ints_n32_kernel (fused imaging, noise, gradients)"
            knote = ("the kernel moves its algorithmic bytes at this rate but is bound by FP32 issue "
                     "(ncu: issue active 61 %, HBM 5 %); compute gives its FFT flop rate")
        roofline = {"kernel": kname, "bound": "hbm",
                    "achieved": ints_gbs, "peak": hbm, "unit": "GB/s", "frac": ints_gbs / hbm,
                    "peak_source": src_note + " hbm_gbs", "traffic": traffic,
                    "note": knote,
                    "algorithmic_bytes_per_launch": ints_bytes,
                    "compute": {"achieved": ints_tf, "peak": fp32_peak, "unit": "TFLOP/s",
                                "frac": ints_tf / fp32_peak,
                                "note": "nominal FFT flops (3 x 5 N^2 log2 N^2 per image) vs nominal FP32 CUDA-core peak"},
                    "raytrace": raytrace}
    p50 = float(np.percentile(step_ms, 50))
    p99 = float(np.percentile(step_ms, 99))
    line = {
        "metric": "subaperture images/s", "value": value, "unit": "subap-images/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": cfg["name"], "wfs": nwfs, "subapertures_per_wfs": wl.nsa,
                   "fft": wl.setup.notf, "pixels": f"{wl.setup.npix}", "layers": nlayer,
                   "screen": f"{cfg['atm']['nx']}^2 FP32", "form": args.form, "noise": True,
                   "gradients": "matched filter" if cfg["phytype"] == 1 else "CoG",
                   "imaging_variant": variant,
                   "l2": "flushed (256 MiB write) before every timed step", "parallelism": f"replicas x{ws}"},
        "frame_latency_ms": {"p50": p50, "p99": p99},
        "stages": st,
        "gpu_launches": int(round(launches_per_step * args.steps)),
        "e2e": {"value": e2e, "unit": "subap-images/s", "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps},
        "roofline": roofline,
        "clocks": clocks,
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(cfg, wl.layers, wl.screens)
        except Exception as e:  # the oracle library may be absent on a foreign host
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    if rank == 0:
        print(json.dumps(line))
    wl.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def run_batch(args, bcfg):
    """The uneven batch: every member's WFS in one frame, replayed as one CUDA graph."""
    import torch
    from maos_b200 import shwfs
    from maos_b200.workload import build_batch
    ws, rank, local = dist_init()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    form = shwfs.SHWFS_FORM_TC if args.form == "tc" else shwfs.SHWFS_FORM_FFT
    wl = build_batch(bcfg["members"], device=local, seed=1 + rank, noisy=True, form=form, graph=True)
    ctx = wl.ctx
    units_per_step = wl.images_per_frame
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    lgs = wl.members[0]
    variant = ctx.autotune(lgs[3][0], lgs[3][-1] + 1, nrep=5)
    isim = 0
    for _ in range(args.warmup):
        wl.frame(isim)
        isim += 1
    ctx.sync()
    barrier(ws, dev)
    clk = ClockSampler(local)
    clk.start()
    time.sleep(0.5)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with torch.cuda.stream(ext):
        for k in range(args.steps):
            flush.zero_()  # L2 flush between timed steps (not timed)
            starts[k].record(ext)
            wl.frame(isim)
            ends[k].record(ext)
            isim += 1
    ctx.sync()
    torch.cuda.synchronize(dev)
    clocks = clk.stop()
    step_ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    tot_ms = allreduce_max(sum(step_ms), ws, dev)
    barrier(ws, dev)
    value = units_per_step * args.steps * ws / (tot_ms * 1e-3)
    # stage timing (stream frames, profiling on; stages summed over the members)
    wl.graph = False
    ctx.profile_enable(True)
    nprof = min(args.steps, 20)
    with torch.cuda.stream(ext):
        for k in range(nprof):
            flush.zero_()
            wl.frame(isim)
            isim += 1
    ctx.sync()
    stages = ctx.profile_read()
    ctx.profile_enable(False)
    wl.graph = True
    launches_per_step = sum(n for _, n in stages.values()) / nprof
    st = {k: dict(ms_per_launch=(ms / n if n else 0.0), launches_per_step=n / nprof, ms_per_step=ms / nprof)
          for k, (ms, n) in stages.items()}
    # end to end: graph frame + host gradients of every WFS into one host buffer
    ctx.copy_counters()
    gbuf = np.empty(sum(2 * ctx.wfs_nsa[i] for i in range(wl.nwfs)))
    e2e_s = 0.0
    for k in range(args.steps):
        with torch.cuda.stream(ext):
            flush.zero_()
        ctx.sync()
        t0 = time.perf_counter()
        wl.frame(isim)
        wl.frame_sync(out=gbuf)
        e2e_s += time.perf_counter() - t0
        isim += 1
    h2d, d2h = ctx.copy_counters()
    e2e_s = allreduce_max(e2e_s, ws, dev)
    e2e = units_per_step * args.steps * ws / e2e_s
    hbm, bf16, src = _peaks()
    lcfg = lgs[0]
    nlayer = len(lcfg["atm"]["ht"])
    ray_bytes = sum(m[1].nsa * len(m[3]) * m[1].nopd ** 2 * (nlayer * 4 + 4) for m in wl.members)
    ray_ms = st["raytrace"]["ms_per_step"]
    ray_gbs = ray_bytes / (ray_ms * 1e-3) / 1e9 if ray_ms else 0.0
    members = [{"workload": m[0]["name"], "wfs": len(m[3]), "subapertures_per_wfs": m[1].nsa,
                "opd_points": m[1].nopd, "fft": m[1].notf, "pixels": m[1].npix} for m in wl.members]
    p50 = float(np.percentile(step_ms, 50))
    p99 = float(np.percentile(step_ms, 99))
    line = {
        "metric": "subaperture images/s", "value": value, "unit": "subap-images/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": bcfg["name"], "members": members, "layers": nlayer,
                   "screen": f"{lcfg['atm']['nx']}^2 FP32", "form": args.form, "noise": True,
                   "frame": "one CUDA graph per frame, one branch per sensor type", "imaging_variant": variant,
                   "l2": "flushed (256 MiB write) before every timed step", "parallelism": f"replicas x{ws}"},
        "frame_latency_ms": {"p50": p50, "p99": p99},
        "stages": st,
        "gpu_launches": int(round(launches_per_step * args.steps)),
        "e2e": {"value": e2e, "unit": "subap-images/s", "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps},
        "roofline": {"kernel": "geom_kernel (ray trace of all members)", "bound": "hbm", "achieved": ray_gbs,
                     "peak": hbm, "unit": "GB/s", "frac": ray_gbs / hbm, "traffic": None,
                     "peak_source": (f"{src} (MEASURED_PEAKS.json) hbm_gbs" if src == "measured" else "fallback"),
                     "algorithmic_bytes_per_step": ray_bytes},
        "clocks": clocks,
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(lcfg, wl.layers, wl.screens)
            line["cpu_baseline"]["sample"] += " (the batch's dominant member)"
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    if rank == 0:
        print(json.dumps(line))
    wl.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def run_serving(args):
    """Serving loop: 32 seeded simulations, Poisson frame requests at a rate sweep."""
    import torch
    from maos_b200 import shwfs
    from maos_b200.serving import Server, draw_sim_cfg, poisson_arrivals
    ws, rank, local = dist_init()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    nsim = 32
    cfgs = [draw_sim_cfg(s) for s in range(nsim)]
    srv = Server(cfgs, device=local, form=shwfs.SHWFS_FORM_FFT, seed=1 + rank)
    srv.prewarm()
    clk = ClockSampler(local)
    clk.start()
    sweeps = {}
    rates = [1000.0, 2000.0, 5000.0, 10000.0, 20000.0]
    for form_name, form in (("fft", shwfs.SHWFS_FORM_FFT), ("tc", shwfs.SHWFS_FORM_TC)):
        srv.set_form(form)
        out = []
        for j, rate in enumerate(rates):
            n = int(min(max(rate * args.serve_seconds, 200), 20000))
            arr = poisson_arrivals(rate, n, nsim, seed=100 + j)
            out.append(srv.run(arr, rate).summary())
        sweeps[form_name] = out
    clocks = clk.stop()
    top = sweeps["fft"][-1]
    resident = len(srv.sims)
    footprint = srv.adm.used
    srv.close()
    line = {
        "metric": "subaperture images/s", "value": top["images_per_s"] * ws, "unit": "subap-images/s",
        "n_gpus": ws, "steps": top["requests"], "warmup": 1, "ms_per_step": top["p50_ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "serving_32sims", "sims": [c["name"] for c in cfgs], "resident": resident,
                   "footprint_bytes": footprint, "rates_req_per_s": rates,
                   "request": "one frame of every WFS of one simulation, gradients to the host",
                   "value": "images/s served at the highest rate, FFT form"},
        "frame_latency_ms": {"p50": top["p50_ms"], "p99": top["p99_ms"]},
        "serving": sweeps,
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line))
    return 0


def _science_ctx(scfg, device, seed):
    import torch  # noqa: F401
    from maos_b200 import shwfs
    from maos_b200.setup import aperture, screens
    from maos_b200.workload import wind
    x, y, a = aperture(scfg["D"], scfg["Din"], scfg["dx"])
    ctx = shwfs.Context(device)
    ctx.set_dt(scfg["dt"])
    at = scfg["atm"]
    n = at["nx"]
    scr = screens(n, n, at["dx"], at["r0"], at["L0"], at["wt"], seed)
    vx, vy = wind(scfg, seed)
    o = -n / 2 * at["dx"]
    layers = [dict(nx=n, ny=n, dx=at["dx"], ox=o, oy=o, ht=float(h), vx=float(vx[i]), vy=float(vy[i]), alpha=1.0)
              for i, h in enumerate(at["ht"])]
    ctx.atm_set(layers, scr)
    ctx.evl_set_aper(x, y, scfg["dx"], a)
    for d in scfg["dirs"]:
        ctx.evl_add_dir(*d)
    ctx.evl_set_psf(scfg["wvl"], scfg["nembed"], scfg["psfsize"], pttr=scfg["pttr"])
    # points traced per direction: the 16x16 tiles that hold aperture points
    X = np.rint((x - x.min()) / scfg["dx"]).astype(np.int64)
    Y = np.rint((y - y.min()) / scfg["dx"]).astype(np.int64)
    ntx = (X.max() + 16) // 16
    traced = 256 * len(np.unique((Y // 16) * ntx + X // 16))
    return ctx, len(x), layers, scr, traced


def science_flops(scfg, nX):
    """Nominal FFT flops of one direction-frame's PSFs: per wavelength nY rows
    and psfsize columns of N-point transforms (5 N log2 N each)."""
    tot = 0.0
    for N, ps in zip(scfg["nembed"], scfg["psfsize"]):
        tot += (nX + ps) * 5 * N * math.log2(N)
    return tot


def science_cpu(scfg, layers, scr, seconds=20.0, max_frames=4):
    from oracle import ref
    e = ref.RefEvl(scfg["D"], scfg["Din"], scfg["dx"], wvl=scfg["wvl"], nembed=scfg["nembed"])
    ref.atm_set(scr, layers)
    t, n = 0.0, 0
    while t < seconds and n < max_frames:
        d = scfg["dirs"][n % len(scfg["dirs"])]
        t0 = time.perf_counter()
        e.frame(d[0], d[1], d[2], n, scfg["dt"], pttr=scfg["pttr"], psfsize=scfg["psfsize"])
        t += time.perf_counter() - t0
        n += 1
    nw = len(scfg["wvl"])
    return n / t, n, min(nw, os.cpu_count() or 1)


def run_science(args, scfg):
    """Science path: every direction of a frame (ray trace, WFE, PSFs)."""
    import torch
    ws, rank, local = dist_init()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if args.impl == "reference":
        if rank != 0:
            return 0
        from maos_b200.setup import screens
        from maos_b200.workload import wind
        at = scfg["atm"]
        n = at["nx"]
        scr = screens(n, n, at["dx"], at["r0"], at["L0"], at["wt"], 1)
        vx, vy = wind(scfg, 1)
        o = -n / 2 * at["dx"]
        layers = [dict(nx=n, ny=n, dx=at["dx"], ox=o, oy=o, ht=float(h), vx=float(vx[i]), vy=float(vy[i]))
                  for i, h in enumerate(at["ht"])]
        v, nfr, cores = science_cpu(scfg, layers, scr, seconds=30.0, max_frames=max(args.steps, 1))
        sample = (f"{nfr} direction-frames of {scfg['name']}: prop of 7 layers onto aper->locs, loc_calc_ptt, "
                  f"locfft_psf at 3 wavelengths (reference C, FFT stand-in for FFTW)")
        print(json.dumps({"impl": "reference", "metric": "science direction-frames/s", "value": v,
                          "unit": "direction-frames/s", "n_gpus": args.gpus, "steps": nfr, "warmup": 0,
                          "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                          "config": {"workload": scfg["name"], "step": "one direction-frame (reference CPU path)"},
                          "cpu_baseline": {"value": v, "unit": "direction-frames/s", "cores": cores,
                                           "kind": "reference", "sample": sample},
                          "e2e": {"value": v, "unit": "direction-frames/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return 0
    ctx, nloc, layers, scr, npts_traced = _science_ctx(scfg, local, 1 + rank)
    nevl = len(scfg["dirs"])
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    isim = 0
    for _ in range(args.warmup):
        ctx.evl_queue(isim, do_psf=True)
        ctx.evl_sync()
        isim += 1
    barrier(ws, dev)
    clk = ClockSampler(local)
    clk.start()
    time.sleep(0.5)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with torch.cuda.stream(ext):
        for k in range(args.steps):
            flush.zero_()
            starts[k].record(ext)
            ctx.evl_queue(isim, do_psf=True)
            ends[k].record(ext)
            isim += 1
    ctx.sync()
    torch.cuda.synchronize(dev)
    clocks = clk.stop()
    step_ms = [s_.elapsed_time(e_) for s_, e_ in zip(starts, ends)]
    tot_ms = allreduce_max(sum(step_ms), ws, dev)
    value = nevl * args.steps * ws / (tot_ms * 1e-3)
    ctx.profile_enable(True)
    nprof = min(args.steps, 10)
    with torch.cuda.stream(ext):
        for k in range(nprof):
            flush.zero_()
            ctx.evl_queue(isim, do_psf=True)
            isim += 1
    ctx.sync()
    stages = ctx.profile_read()
    ctx.profile_enable(False)
    launches_per_step = sum(n for _, n in stages.values()) / nprof
    ctx.copy_counters()
    e2e_s = 0.0
    for k in range(args.steps):
        with torch.cuda.stream(ext):
            flush.zero_()
        ctx.sync()
        t0 = time.perf_counter()
        ctx.evl_queue(isim, do_psf=True)
        ctx.evl_sync()
        e2e_s += time.perf_counter() - t0
        isim += 1
    h2d, d2h = ctx.copy_counters()
    e2e_s = allreduce_max(e2e_s, ws, dev)
    e2e = nevl * args.steps * ws / e2e_s
    st = {k: dict(ms_per_launch=(ms / n if n else 0.0), launches_per_step=n / nprof, ms_per_step=ms / nprof)
          for k, (ms, n) in stages.items()}
    hbm, bf16, src = _peaks()
    src_note = f"{src} (MEASURED_PEAKS.json)" if src == "measured" else "fallback"
    nlayer = len(scfg["atm"]["ht"])
    ray_bytes = nevl * npts_traced * (nlayer * 4 + 4)
    ray_ms = st["raytrace"]["ms_per_step"]
    ray_gbs = ray_bytes / (ray_ms * 1e-3) / 1e9 if ray_ms else 0.0
    psf_ms = st["ints"]["ms_per_step"]
    nX = int(round(scfg["D"] / scfg["dx"])) + 3
    psf_flops = nevl * science_flops(scfg, nX)
    fp32_peak = 148 * 128 * 2 * 1.965e9 / 1e12
    psf_tf = psf_flops / (psf_ms * 1e-3) / 1e12 if psf_ms else 0.0
    roofline = {"kernel": "geom_kernel (aperture ray trace)", "bound": "hbm", "achieved": ray_gbs, "peak": hbm,
                "unit": "GB/s", "frac": ray_gbs / hbm, "peak_source": src_note + " hbm_gbs", "traffic": None,
                "algorithmic_bytes_per_launch": ray_bytes,
                "psf": {"kernels": "evl_psf_rows_kernel + evl_psf_cols_kernel", "achieved": psf_tf,
                        "peak": fp32_peak, "unit": "TFLOP/s", "frac": psf_tf / fp32_peak,
                        "flops_per_step": psf_flops,
                        "note": "nominal FFT flops (5 N log2 N per transform, pruned rows and columns) vs "
                                "nominal FP32 CUDA-core peak"}}
    line = {
        "metric": "science direction-frames/s", "value": value, "unit": "direction-frames/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": scfg["name"], "directions": nevl, "aperture_points": nloc,
                   "wavelengths": scfg["wvl"], "psf_grid": scfg["nembed"], "psf_size": scfg["psfsize"],
                   "layers": nlayer, "screen": f"{scfg['atm']['nx']}^2 FP32",
                   "l2": "flushed (256 MiB write) before every timed step", "parallelism": f"replicas x{ws}"},
        "stages": st,
        "gpu_launches": int(round(launches_per_step * args.steps)),
        "e2e": {"value": e2e, "unit": "direction-frames/s", "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps},
        "roofline": roofline,
        "clocks": clocks,
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            v, nfr, cores = science_cpu(scfg, layers, scr)
            line["cpu_baseline"] = {"value": v, "unit": "direction-frames/s", "cores": cores, "kind": "reference",
                                    "sample": f"{nfr} direction-frames: prop onto aper->locs, loc_calc_ptt, "
                                              f"locfft_psf at 3 wavelengths (reference C, FFT stand-in)"}
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="lgs30_6x60x60_mf")
    ap.add_argument("--form", default="fft", choices=["fft", "tc"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-seconds", type=float, default=0.5, help="serving: seconds of requests per rate")
    args = ap.parse_args()
    from maos_b200.configs import CONFIGS, BATCHES, SCIENCE
    if args.warmup < 3:
        args.warmup = 3
    if args.config in SCIENCE:
        return run_science(args, SCIENCE[args.config])
    if args.config == "serving_32sims":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no serving loop"}))
            return 0
        return run_serving(args)
    if args.config in BATCHES:
        bcfg = BATCHES[args.config]
        if args.impl == "reference":
            return run_reference(args, bcfg["members"][0])
        return run_batch(args, bcfg)
    cfg = CONFIGS[args.config]
    if args.impl == "reference":
        return run_reference(args, cfg)
    return run_b200(args, cfg)


if __name__ == "__main__":
    sys.exit(main())
