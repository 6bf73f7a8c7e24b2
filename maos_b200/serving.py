"""Serving loop: frame requests from many independent simulations on one GPU.

Each simulation (sim) is a complete Shack-Hartmann setup drawn from a seed
(telescope diameter, subaperture order, WFS count, FFT size, layer count);
its screens, transfer functions and gradient operators stay resident in HBM
in its own context and CUDA stream.  Requests arrive as a Poisson stream.
The loop is continuous batching: every request whose sim is resident and idle
is launched at once, whatever else is on the device, so the frames of
different sims overlap; completions are polled from CUDA events.  Sims are
admitted by their measured device footprint against an HBM budget, in the
order their first request arrives; an admitted sim with no queued or running
work may be evicted to admit a waiting one.

Latency of a request = time from its (scheduled) arrival to the host seeing
its gradients, queueing included.
"""
from __future__ import annotations

import collections
import math
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional

import numpy as np

from .configs import AS2RAD


# ---------------------------------------------------------------------------
# simulations drawn from a seed
# ---------------------------------------------------------------------------
_HT = [0.0, 500.0, 1e3, 2e3, 4e3, 8e3, 16e3]
_WT = [0.596, 0.0386, 0.0386, 0.0386, 0.1436, 0.0386, 0.1024]


def draw_sim_cfg(seed: int, screen_nx: int = 1024) -> dict:
    """One simulation's configuration: D in {8, 10, 30} m, order in {16, 32, 60},
    1-6 NGS WFS, FFT in {32, 64} (16 or 32 OPD points per subaperture), 2-7 layers
    with r0 = 0.186 m, L0 = 30 m; CoG gradients, 8x8 Nyquist pixels."""
    rng = np.random.default_rng(1000 + seed)
    D = float(rng.choice([8.0, 10.0, 30.0]))
    order = int(rng.choice([16, 32, 60]))
    notf = int(rng.choice([32, 64]))
    nwfs = int(rng.integers(1, 7))
    nl = int(rng.integers(2, 8))
    nopd = notf // 2
    dsa = D / order
    wvl = 0.7e-6
    wt = np.asarray(_WT[:nl])
    wt = list(wt / wt.sum())
    ang = rng.uniform(0, 2 * math.pi, nwfs)
    rad = rng.uniform(0, 30.0, nwfs) * AS2RAD
    return dict(
        name=f"sim{seed}_D{D:g}_o{order}_w{nwfs}_f{notf}_l{nl}",
        D=D, Din=0.12 * D, amp_binary=0,
        order=order, dsa=dsa, dx=dsa / nopd, saat=0.3, embfac=2, notf=notf,
        pixpsa=8, pixtheta=0.5 * wvl / dsa, pixblur=0.3, wvl=wvl, hs=math.inf,
        siglev=1000.0, rne=3.0, bkgrnd=0.0, bkgrndc=0.0,
        phytype=2, sigmatch=1, mtchcr=0, cogthres=0.0, cogoff=0.0,
        r0=0.186, L0=30.0, has_llt=0, nwfs=nwfs,
        thetax=list(rad * np.cos(ang)), thetay=list(rad * np.sin(ang)),
        atm=dict(r0=0.186, L0=30.0, nx=screen_nx, dx=1.0 / 32, ht=_HT[:nl], wt=wt,
                 ws=list(rng.uniform(5.0, 15.0, nl)), wdir_deg=list(rng.uniform(0, 360.0, nl))),
        dt=1.0 / 800,
    )


def poisson_arrivals(rate: float, n: int, nsim: int, seed: int):
    """n requests: (arrival time in s, sim index), exponential gaps at `rate`."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    return list(zip(t.tolist(), rng.integers(0, nsim, n).tolist()))


# ---------------------------------------------------------------------------
# admission by footprint
# ---------------------------------------------------------------------------
class Admission:
    """Which sims are resident.  load(i) makes sim i resident and returns its
    device footprint in bytes; unload(i) frees it.  A sim is admitted when its
    footprint (known after a first load, else the estimate) fits the budget,
    evicting idle resident sims (least recently used first) if needed."""

    def __init__(self, budget: int, load: Callable[[int], int], unload: Callable[[int], None],
                 estimate: Callable[[int], int]):
        self.budget = budget
        self._load, self._unload, self._estimate = load, unload, estimate
        self.resident: "collections.OrderedDict[int, int]" = collections.OrderedDict()  # sim -> bytes
        self.known: Dict[int, int] = {}
        self.evictions = 0

    @property
    def used(self) -> int:
        return sum(self.resident.values())

    def touch(self, i: int):
        self.resident.move_to_end(i)

    def try_admit(self, i: int, busy) -> bool:
        """Admit sim i if it fits, evicting resident sims not in `busy`."""
        if i in self.resident:
            self.touch(i)
            return True
        need = self.known.get(i, self._estimate(i))
        if need > self.budget:
            return False
        while self.used + need > self.budget:
            victim = next((j for j in self.resident if j not in busy), None)
            if victim is None:
                return False
            self._unload(victim)
            del self.resident[victim]
            self.evictions += 1
        got = self._load(i)
        self.known[i] = got
        self.resident[i] = got
        return True


# ---------------------------------------------------------------------------
# the loop
# ---------------------------------------------------------------------------
@dataclass
class Stats:
    rate: float
    latencies_ms: List[float] = field(default_factory=list)
    images: int = 0
    wall_s: float = 0.0
    evictions: int = 0

    def summary(self) -> dict:
        lat = np.asarray(self.latencies_ms) if self.latencies_ms else np.zeros(1)
        return {"rate_req_per_s": self.rate, "requests": len(self.latencies_ms),
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "frames_per_s": len(self.latencies_ms) / self.wall_s if self.wall_s else 0.0,
                "images_per_s": self.images / self.wall_s if self.wall_s else 0.0,
                "evictions": self.evictions}


class Server:
    """Continuous-batching frame server over independent simulations on one GPU."""

    def __init__(self, cfgs: List[dict], device: int = 0, form: int = 0, hbm_budget: Optional[int] = None,
                 seed: int = 1, priority: Optional[str] = None):
        import torch
        from . import shwfs
        from .setup import Setup
        self.torch = torch
        self.cfgs = cfgs
        self.device = device
        self.form = form
        self.seed = seed
        self.setups = [Setup(c) for c in cfgs]  # host setup of every sim, ahead of time
        self.priority = priority
        self.sims: Dict[int, object] = {}
        self.isim = [0] * len(cfgs)
        free, total = torch.cuda.mem_get_info(device)
        budget = hbm_budget if hbm_budget is not None else int(0.8 * free)
        self.adm = Admission(budget, self._load, self._unload, self._estimate)
        self._shwfs = shwfs

    def _estimate(self, i: int) -> int:
        c, s = self.cfgs[i], self.setups[i]
        nl, nx = len(c["atm"]["ht"]), c["atm"]["nx"]
        per_img = s.nopd ** 2 * 8 + s.npix * 4 + (s.notf ** 2 * 8 if s.notf != 32 else 0)
        return nl * nx * nx * 4 + c["nwfs"] * s.nsa * per_img + (64 << 20)

    def cost(self, i: int) -> float:
        """Relative device work of one frame of sim i: images x FFT points x log2 of the points."""
        c, s = self.cfgs[i], self.setups[i]
        n = s.notf
        return c["nwfs"] * s.nsa * n * n * math.log2(n)

    def stream_priority(self, i: int) -> int:
        """CUDA stream priority of sim i under the server's policy (lower runs first):
        "large" gives the costliest frames the greatest priority, in equal steps of the
        cost's logarithm over the device's levels; "small" the reverse; None all 0."""
        if self.priority is None:
            return 0
        lo, hi = self.torch.cuda.Stream.priority_range() if hasattr(self.torch.cuda.Stream, "priority_range") \
            else (0, -5)
        levels = lo - hi
        cmin = min(self.cost(j) for j in range(len(self.cfgs)))
        cmax = max(self.cost(j) for j in range(len(self.cfgs)))
        f = math.log(self.cost(i) / cmin) / math.log(cmax / cmin) if cmax > cmin else 0.0
        if self.priority == "small":
            f = 1.0 - f
        return lo - int(round(f * levels))

    def _load(self, i: int) -> int:
        from .workload import build_from_setup
        torch = self.torch
        torch.cuda.synchronize(self.device)
        f0 = torch.cuda.mem_get_info(self.device)[0]
        wl = build_from_setup(self.cfgs[i], self.setups[i], device=self.device, seed=self.seed + i, noisy=True,
                              form=self.form)
        if self.priority is not None:
            wl.ctx.set_stream_priority(self.stream_priority(i))
        ext = torch.cuda.ExternalStream(wl.ctx.stream, device=self.device)
        # one host buffer per sim: a request's gradients land there, with no
        # allocation per request (copied out only when a caller keeps results)
        gbuf = np.empty(sum(2 * wl.ctx.wfs_nsa[k] for k in wl.wfs))
        self.sims[i] = (wl, ext, torch.cuda.Event(), gbuf)
        wl.frame(0)  # buffers made on first use belong to the footprint too
        wl.frame_sync()
        torch.cuda.synchronize(self.device)
        return max(f0 - torch.cuda.mem_get_info(self.device)[0], 1)

    def _unload(self, i: int):
        wl, _, _, _ = self.sims.pop(i)
        wl.ctx.close()

    def prewarm(self):
        """Admit the sims that fit, in index order (each load runs a first
        frame, so no allocation happens in a timed run)."""
        for i in range(len(self.cfgs)):
            self.adm.try_admit(i, busy=set(self.sims))

    def set_form(self, form: int):
        """Imaging form of every resident sim (and of sims loaded later); one
        frame per sim builds what the form needs before anything is timed."""
        self.form = form
        for i, (wl, _, _, _) in self.sims.items():
            wl.ctx.set_form(form)
            wl.frame(0)
            wl.frame_sync()

    def launch(self, i: int, isim: int):
        wl, ext, ev, _ = self.sims[i]
        wl.frame(isim)
        ev.record(ext)

    def done(self, i: int) -> bool:
        return self.sims[i][2].query()

    def collect(self, i: int, keep: bool = False):
        """The gradients of sim i's finished request, in its host buffer; with keep, a copy
        split per WFS."""
        wl, _, _, gbuf = self.sims[i]
        wl.frame_sync(out=gbuf)
        if not keep:
            return gbuf
        sizes = [2 * wl.ctx.wfs_nsa[k] for k in wl.wfs]
        return [a.copy() for a in np.split(gbuf, np.cumsum(sizes)[:-1])]

    def run(self, arrivals, rate: float, results: Optional[dict] = None) -> Stats:
        """Serve `arrivals` [(t, sim)] in real time; returns latency statistics.
        With `results`, each request's [(grad, ints)] per WFS is kept under
        (sim, frame index)."""
        st = Stats(rate=rate)
        pending = collections.deque(arrivals)
        waiting: Dict[int, collections.deque] = collections.defaultdict(collections.deque)
        order: "collections.OrderedDict[int, None]" = collections.OrderedDict()  # sims with waiting requests
        inflight: Dict[int, float] = {}  # sim -> arrival time of its running request
        running: Dict[int, int] = {}     # sim -> frame index of its running request
        t0 = time.perf_counter()

        def launch_ready():
            # every waiting request whose sim is idle goes to the device now
            for i in list(order):
                if i in inflight:
                    continue
                if i in self.adm.resident:
                    self.adm.touch(i)
                elif not self.adm.try_admit(i, busy=set(inflight) | set(order)):
                    continue
                t = waiting[i].popleft()
                if not waiting[i]:
                    del order[i]
                self.launch(i, self.isim[i])
                running[i] = self.isim[i]
                self.isim[i] += 1
                inflight[i] = t

        while pending or order or inflight:
            now = time.perf_counter() - t0
            while pending and pending[0][0] <= now:
                t, i = pending.popleft()
                waiting[i].append(t)
                order.setdefault(i, None)
            # launches first, so that new work reaches the device before the host
            # spends time collecting finished frames
            launch_ready()
            finished = [j for j in inflight if self.done(j)]
            for i in finished:
                out = self.collect(i, keep=results is not None)
                if results is not None:
                    results[(i, running[i])] = out
                st.latencies_ms.append(1e3 * (time.perf_counter() - t0 - inflight.pop(i)))
                st.images += self.cfgs[i]["nwfs"] * self.setups[i].nsa
            if finished:
                launch_ready()
            if not inflight and pending and not order:
                time.sleep(max(0.0, min(pending[0][0] - (time.perf_counter() - t0), 1e-3)))
        st.wall_s = time.perf_counter() - t0
        st.evictions = self.adm.evictions
        return st

    def close(self):
        for i in list(self.sims):
            self._unload(i)
        for s in self.setups:
            s.close()
