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

_OUT_FD = None


def emit(line: dict):
    """Write the one JSON result line to the real standard output.  Everything
    else the process writes to file descriptor 1 (the reference library's
    progress messages included) goes to standard error."""
    fd = _OUT_FD if _OUT_FD is not None else 1
    os.write(fd, (json.dumps(line) + "\n").encode())


def _stdout_to_stderr():
    global _OUT_FD
    sys.stdout.flush()
    _OUT_FD = os.dup(1)
    os.dup2(2, 1)


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


FFT_BACKEND = ("the oracle's FFT stand-in (oracle/refbuild/fftw_standin.c, FFTW's conventions in double): "
               "FFTW is absent from this image (no libfftw3 in the dynamic linker cache)")


def ref_frame(r, cfg, isim, seed, noisy=True):
    """One frame of every WFS of the config on the reference's CPU path; seconds."""
    from oracle import ref
    dt = cfg.get("dt", 1.0 / 800)
    return sum(ref.frame_full_mt(r, iwfs, isim, dt, seed=seed * 1000003 + iwfs, noisy=noisy)[2]
               for iwfs in range(cfg["nwfs"]))


def ref_workload(cfg, seed=1):
    """The reference's own setup and screens of a config (oracle/_ref only):
    RefPowfs (maos/powfs.c setup), genscreen (lib/turbulence.c) and the same
    winds as the B200 arm."""
    from oracle import ref
    from maos_b200.configs import layers_of
    ncpu = os.cpu_count() or 1
    r = ref.RefPowfs(cfg, nthread=ncpu)
    a = cfg["atm"]
    scr = ref.genscreen(a["nx"], a["nx"], a["dx"], a["r0"], a["L0"], a["wt"], seed)
    ref.atm_set(scr, layers_of(cfg, seed))
    return r, ncpu


def cpu_baseline(cfg, wl_layers, screens, seconds=15.0, max_frames=40):
    """The reference's CPU frame of every WFS, timed on this host's cores for a
    bounded sample of frames (about `seconds` of CPU work)."""
    from oracle import ref
    ncpu = os.cpu_count() or 1
    r = ref.RefPowfs(cfg, nthread=ncpu)
    ref.atm_set(screens, wl_layers)
    ref_frame(r, cfg, 0, 1)  # warm plans and caches
    t = 0.0
    n = 0
    while t < seconds and n < max_frames:
        t += ref_frame(r, cfg, n + 1, n + 1)
        n += 1
    return {"value": r.nsa * cfg["nwfs"] * n / t, "unit": "subap-images/s", "cores": ncpu, "kind": "reference",
            "fft_backend": FFT_BACKEND,
            "sample": f"{n} frames of all {cfg['nwfs']} WFS of {cfg['name']} ({r.nsa} subapertures each): 7-layer "
                      f"ray trace, LLT uplink, wfsints, addnoise, matched filter; reference C (oracle/_ref), "
                      f"NTHREAD={ncpu}"}


def run_reference(args, cfg):
    """The reference's own CPU path (oracle/_ref: its maos/lib/math/sys C) on the
    same workload and config as the B200 arm: one step is one frame of every
    WFS.  Loads no library of this repository."""
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    from oracle import ref
    from maos_b200.configs import workload_desc
    if not ref.available():
        emit({"impl": "reference", "unavailable": "oracle/_ref/libmaosref.so is not built"})
        return 0
    r, ncpu = ref_workload(cfg, seed=1)
    for i in range(args.warmup):
        ref_frame(r, cfg, i, i + 1)
    times = [ref_frame(r, cfg, args.warmup + k, k + 7) for k in range(args.steps)]
    tot = sum(times)
    units = r.nsa * cfg["nwfs"]
    value = units * args.steps / tot
    line = {
        "impl": "reference", "metric": "subaperture images/s", "value": value, "unit": "subap-images/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_desc(cfg, r.nsa, r.notf, r.npix),
        "cpu_baseline": {"value": value, "unit": "subap-images/s", "cores": ncpu, "kind": "reference",
                         "fft_backend": FFT_BACKEND,
                         "sample": f"{args.steps} frames of all {cfg['nwfs']} WFS of {cfg['name']} "
                                   f"({r.nsa} subapertures each), NTHREAD={ncpu}"},
        "e2e": {"value": value, "unit": "subap-images/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    emit(line)
    return 0


def _time_frames(wl, ext, flush, isim, steps):
    """Device time of `steps` frames (CUDA events on the context stream, L2
    flushed before each, the flush untimed); returns (per-step ms, next isim)."""
    import torch
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    with torch.cuda.stream(ext):
        for k in range(steps):
            flush.zero_()  # L2 flush between timed steps (not timed)
            starts[k].record(ext)
            wl.frame(isim)
            ends[k].record(ext)
            isim += 1
    wl.ctx.sync()
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in zip(starts, ends)], isim


def _stage_profile(wl, ext, flush, isim, nprof):
    """Per-stage device time of nprof frames (stage events on, separate from the timed frames)."""
    import torch
    ctx = wl.ctx
    ctx.profile_enable(True)
    with torch.cuda.stream(ext):
        for k in range(nprof):
            flush.zero_()
            wl.frame(isim)
            isim += 1
    ctx.sync()
    stages = ctx.profile_read()
    ctx.profile_enable(False)
    st = {k: dict(ms_per_launch=(ms / n if n else 0.0), launches_per_step=n / nprof, ms_per_step=ms / nprof)
          for k, (ms, n) in stages.items()}
    return st, sum(n for _, n in stages.values()) / nprof, isim


def _roofline(form, cfg, wl, st, units_per_step):
    """Roofline of the form's dominant kernel from its live per-launch time."""
    hbm, bf16, src = _peaks()
    src_note = f"{src} (MEASURED_PEAKS.json)" if src == "measured" else "fallback"
    nwfs = len(wl.wfs)
    nlayer = len(cfg["atm"]["ht"])
    ints_bytes, ray_bytes = algorithmic_traffic(cfg, wl.nsa, wl.npix, wl.setup.nopd, wl.setup.notf, nwfs, nlayer)
    ints_ms = st["ints"]["ms_per_launch"]
    ray_ms = st["raytrace"]["ms_per_step"]  # the WFS pupils, plus any LLT pupils traced in a second launch
    ints_gbs = ints_bytes / (ints_ms * 1e-3) / 1e9 if ints_ms else 0.0
    ray_gbs = ray_bytes / (ray_ms * 1e-3) / 1e9 if ray_ms else 0.0
    measured = {}
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            measured = json.load(f)
    traffic = measured.get(f"{cfg['name']}:{form}:ints")
    raytrace = {"kernel": "geom_kernel", "bound": "hbm", "achieved": ray_gbs, "peak": hbm, "unit": "GB/s",
                "frac": ray_gbs / hbm, "algorithmic_bytes_per_launch": ray_bytes,
                "traffic": measured.get(f"{cfg['name']}:raytrace"),
                "limiter": "L1/L2 gather latency: the measured DRAM bytes (traffic, one launch of the WFS pupils) "
                           "are a fraction of the algorithmic bytes, each touched screen byte crossing from DRAM "
                           "about once",
                "note": "algorithmic bytes: one 4-byte screen read per point and layer plus the OPD write"}
    hbm_sub = {"achieved": ints_gbs, "peak": hbm, "unit": "GB/s", "frac": ints_gbs / hbm,
               "peak_source": src_note + " hbm_gbs", "algorithmic_bytes_per_launch": ints_bytes}
    if form == "tc":
        tflops = units_per_step * tc_mma_flops_per_image() / (ints_ms * 1e-3) / 1e12 if ints_ms else 0.0
        return {"kernel": "ints_tc_kernel (tcgen05 BF16x3 DFT imaging)", "bound": "tensor",
                "achieved": tflops, "peak": bf16, "unit": "TFLOP/s", "frac": tflops / bf16,
                "peak_source": src_note + " bf16_tflops, burst", "traffic": traffic,
                "flops_per_launch": units_per_step * tc_mma_flops_per_image(),
                "hbm": hbm_sub, "post": {"kernel": "noise_grad_kernel", "ms_per_launch": st["post"]["ms_per_launch"]},
                "raytrace": raytrace}
    flops = fft_flops_per_image(wl.setup.notf) * units_per_step
    fp32_peak = 148 * 128 * 2 * 1.965e9 / 1e12  # nominal FP32 CUDA-core peak, TFLOP/s
    ints_tf = flops / (ints_ms * 1e-3) / 1e12 if ints_ms else 0.0
    if wl.setup.notf == 64:
        kname = "ints_n64_kernel (fused imaging, noise, gradients; half-spectrum transforms)"
    else:
        kname = "ints_n32_kernel (fused imaging, noise, gradients)"
    return {"kernel": kname, "bound": "fp32", "achieved": ints_tf, "peak": fp32_peak, "unit": "TFLOP/s",
            "frac": ints_tf / fp32_peak, "traffic": traffic,
            "peak_source": "nominal FP32 CUDA-core peak (148 SM x 128 lanes x 2 x 1.965 GHz); no measured FP32 peak",
            "flops_per_launch": flops,
            "note": "nominal FFT flops (3 x 5 N^2 log2 N^2 per image); the kernel issues FP32 work and moves its "
                    "algorithmic bytes well below the HBM roof (sub-object hbm)",
            "hbm": hbm_sub, "raytrace": raytrace}


def run_b200(args, cfg):
    """Both imaging forms on one workload: the plain FP32 FFT form and the
    tensor-core BF16x3 DFT form; the line's value is the faster form's."""
    import torch
    from maos_b200 import shwfs
    from maos_b200.configs import workload_desc
    from maos_b200.workload import build
    ws, rank, local = dist_init()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    wl = build(cfg, device=local, seed=1 + rank, noisy=True, form=shwfs.SHWFS_FORM_FFT)
    ctx = wl.ctx
    nwfs = len(wl.wfs)
    units_per_step = nwfs * wl.nsa
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    if args.variant is None:
        variant = ctx.autotune(wl.wfs[0], wl.wfs[-1] + 1, nrep=5)
    else:  # a fixed imaging variant (profiling one kernel)
        variant = args.variant
        ctx.set_variant(wl.ipowfs, variant)
    forms = [args.form] if args.form != "both" else ["fft", "tc"]
    if wl.setup.notf != 32 and "tc" in forms:
        # the tensor-core form is built for the 32-point transforms only; a larger
        # powfs runs the FFT form whichever form is asked for
        forms = ["fft"]
    isim = 0
    res = {}
    clk = ClockSampler(local)
    clk.start()
    for form in forms:
        ctx.set_form(shwfs.SHWFS_FORM_TC if form == "tc" else shwfs.SHWFS_FORM_FFT)
        for _ in range(args.warmup):
            wl.frame(isim)
            isim += 1
        ctx.sync()
        barrier(ws, dev)
        if not res:
            time.sleep(0.5)
        step_ms, isim = _time_frames(wl, ext, flush, isim, args.steps)
        tot_ms = allreduce_max(sum(step_ms), ws, dev)
        barrier(ws, dev)
        st, lps, isim = _stage_profile(wl, ext, flush, isim, min(args.steps, 20))
        res[form] = dict(value=units_per_step * args.steps * ws / (tot_ms * 1e-3), tot_ms=tot_ms, step_ms=step_ms,
                         stages=st, launches_per_step=lps, roofline=_roofline(form, cfg, wl, st, units_per_step))
    clocks = clk.stop()
    best = max(forms, key=lambda f: res[f]["value"])
    ctx.set_form(shwfs.SHWFS_FORM_TC if best == "tc" else shwfs.SHWFS_FORM_FFT)
    # end to end through the C ABI in the headline form: queue + sync with host
    # gradients each step, into one host buffer the loop owns (as a C caller passes its own)
    for _ in range(args.warmup):
        wl.frame(isim)
        isim += 1
    wl.frame_sync()
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
    head = res[best]
    line = {
        "metric": "subaperture images/s", "value": head["value"], "unit": "subap-images/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["tot_ms"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_desc(cfg, wl.nsa, wl.setup.notf, wl.npix),
        "form": best, "imaging_variant": variant, "noise": True,
        "l2": "flushed (256 MiB write) before every timed step", "parallelism": f"replicas x{ws}",
        "frame_latency_ms": {"p50": float(np.percentile(head["step_ms"], 50)),
                             "max": float(np.max(head["step_ms"])),
                             "note": "device time per frame over the timed steps (the serving loop's p99 is its own "
                                     "bench mode)"},
        "stages": head["stages"],
        "gpu_launches": int(round(head["launches_per_step"] * args.steps)),
        "e2e": {"value": e2e, "unit": "subap-images/s", "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps, "form": best},
        "roofline": head["roofline"],
        "clocks": clocks,
    }
    if len(forms) == 2:
        line["forms"] = {f: {"value": res[f]["value"], "ms_per_step": res[f]["tot_ms"] / args.steps,
                             "stages": res[f]["stages"], "roofline": res[f]["roofline"]} for f in forms}
        line["tc_over_fft"] = res["tc"]["value"] / res["fft"]["value"]
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(cfg, wl.layers, wl.screens)
        except Exception as e:  # the oracle library may be absent on a foreign host
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    if rank == 0:
        emit(line)
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
    form_name = "tc" if args.form == "tc" else "fft"
    form = shwfs.SHWFS_FORM_TC if form_name == "tc" else shwfs.SHWFS_FORM_FFT
    wl = build_batch(bcfg["members"], device=local, seed=1 + rank, noisy=True, form=form, graph=True)
    ctx = wl.ctx
    units_per_step = wl.images_per_frame
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    lgs = wl.members[0]
    variant = ctx.autotune(lgs[3][0], lgs[3][-1] + 1, nrep=5)
    # both frame layouts: the per-powfs launches (a graph branch per sensor type) and
    # the imaging of all sensors as one persistent work-list launch
    isim = 1000
    layouts = {}
    for name, on in (("branches", False), ("worklist", True)):
        ctx.set_worklist(on)
        for _ in range(args.warmup):
            wl.frame(isim)
            isim += 1
        ctx.sync()
        ms, isim = _time_frames(wl, ext, flush, isim, args.steps)
        layouts[name] = {"value": units_per_step * args.steps / (sum(ms) * 1e-3), "ms_per_step": sum(ms) / args.steps}
    choice = ctx.autotune_frame(0, wl.nwfs, nrep=5)
    layouts["chosen"] = "branches" if choice == 0 else "worklist"
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
                   "screen": f"{lcfg['atm']['nx']}^2 FP32", "form": form_name, "noise": True,
                   "frame": ("one CUDA graph per frame, one branch per sensor type" if choice == 0 else
                             "one CUDA graph per frame: ray traces, then one persistent work-list imaging launch"),
                   "imaging_variant": variant, "layout_choice": choice,
                   "l2": "flushed (256 MiB write) before every timed step", "parallelism": f"replicas x{ws}"},
        "frame_latency_ms": {"p50": p50, "p99": p99},
        "layouts": layouts,
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
        emit(line)
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
        emit(line)
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
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        from oracle import ref
        from maos_b200.configs import layers_of
        at = scfg["atm"]
        n = at["nx"]
        scr = ref.genscreen(n, n, at["dx"], at["r0"], at["L0"], at["wt"], 1)
        layers = layers_of(scfg, 1)
        v, nfr, cores = science_cpu(scfg, layers, scr, seconds=30.0, max_frames=max(args.steps, 1))
        sample = (f"{nfr} direction-frames of {scfg['name']}: prop of 7 layers onto aper->locs, loc_calc_ptt, "
                  f"locfft_psf at 3 wavelengths (reference C, FFT stand-in for FFTW)")
        emit({"impl": "reference", "metric": "science direction-frames/s", "value": v,
              "unit": "direction-frames/s", "n_gpus": args.gpus, "steps": nfr, "warmup": 0,
              "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
              "vs_baseline": None, "dtype": "f64", "data": "synthetic",
              "config": {"workload": scfg["name"], "step": "one direction-frame (reference CPU path)"},
              "cpu_baseline": {"value": v, "unit": "direction-frames/s", "cores": cores,
                               "kind": "reference", "sample": sample},
              "e2e": {"value": v, "unit": "direction-frames/s", "h2d_bytes_per_step": 0,
                      "d2h_bytes_per_step": 0}})
        return 0
    import torch
    ws, rank, local = dist_init()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
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
        emit(line)
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
    ap.add_argument("--form", default="both", choices=["both", "fft", "tc"],
                    help="imaging form(s) to time; both: the FFT and tensor-core forms, value = the faster")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--variant", type=int, default=None,
                    help="imaging-kernel variant of the 32-point FFT form (default: the autotuner's choice)")
    ap.add_argument("--serve-seconds", type=float, default=0.5, help="serving: seconds of requests per rate")
    args = ap.parse_args()
    _stdout_to_stderr()
    from maos_b200.configs import CONFIGS, BATCHES, SCIENCE
    if args.warmup < 3:
        args.warmup = 3
    if args.config in SCIENCE:
        return run_science(args, SCIENCE[args.config])
    if args.config == "serving_32sims":
        if args.impl == "reference":
            emit({"impl": "reference", "unavailable": "the reference has no serving loop"})
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
