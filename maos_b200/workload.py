"""Assemble a complete Shack-Hartmann simulation on one device from a config.

:func:`build` runs the host setup (maos_b200.setup), makes the von Karman
screens with seeded wind directions, declares every WFS and loads the matched
filter; the returned :class:`Workload` runs frames through the C ABI.  It is
the standalone counterpart of the reference's maos_setup + gpu_wfsgrad_init +
gpu_atm2gpu sequence (maos/setup.c:56-203, maos/sim.c:79).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List

import numpy as np

from . import shwfs
from .configs import layers_of, wind  # noqa: F401  (wind is re-exported)
from .setup import Setup, screens


@dataclass
class Workload:
    cfg: dict
    ctx: "shwfs.Context"
    setup: Setup
    ipowfs: int
    wfs: List[int]
    layers: List[dict] = field(default_factory=list)
    screens: List[np.ndarray] = field(default_factory=list)

    @property
    def nsa(self) -> int:
        return self.setup.nsa

    @property
    def npix(self) -> int:
        return self.setup.npix

    def frame(self, isim: int):
        """Queue one frame of every WFS (asynchronous)."""
        self.ctx.frame_queue(isim, self.wfs[0], self.wfs[-1] + 1)

    def frame_sync(self, want_ints: bool = False, out=None):
        """Gradients of every WFS with one wait (one array per WFS, or all of
        them written into ``out``: see Context.frame_sync_range); with
        want_ints, (gradients, intensities) per WFS."""
        if not want_ints:
            return self.ctx.frame_sync_range(self.wfs[0], self.wfs[-1] + 1, out=out)
        return [self.ctx.frame_sync(i, self.ipowfs, want_ints) for i in self.wfs]

    def close(self):
        self.ctx.close()
        self.setup.close()


def build(cfg: dict, device: int = 0, seed: int = 1, noisy: bool = True, nx: int = None,
          form: int = shwfs.SHWFS_FORM_FFT) -> Workload:
    return build_from_setup(cfg, Setup(cfg), device=device, seed=seed, noisy=noisy, nx=nx, form=form)


def build_from_setup(cfg: dict, setup: Setup, device: int = 0, seed: int = 1, noisy: bool = True, nx: int = None,
                     form: int = shwfs.SHWFS_FORM_FFT) -> Workload:
    """As build, from a host setup made beforehand (which the workload then owns)."""
    ctx = shwfs.Context(device)
    ctx.set_form(form)
    ctx.set_dt(cfg.get("dt", 1.0 / 800))
    ip = setup.load(ctx)
    # further wavelengths (cfg["wvls"][1:], weights cfg["wvlwts"]): one band each, set up at its wavelength
    wvls = list(cfg.get("wvls", [cfg["wvl"]]))
    wts = list(cfg.get("wvlwts", [1.0] * len(wvls)))
    for wv, wt in zip(wvls[1:], wts[1:]):
        sb = Setup(dict(cfg, wvl=wv))
        sb.load_band(ctx, ip, wt)
        sb.close()
    wl = []
    for k in range(cfg["nwfs"]):
        i = ctx.wfs_add(ipowfs=ip, thetax=cfg["thetax"][k], thetay=cfg["thetay"][k], hs=cfg["hs"], hc=0.0,
                        misregx=0.0, misregy=0.0, sigsim=cfg["siglev"], wvlwt=wts[0], noisy=1 if noisy else 0)
        setup.load_wfs(ctx, i)
        ctx.wfs_seed(i, seed * 1000003 + k)
        wl.append(i)
    a = cfg["atm"]
    n = nx or a["nx"]
    scr = screens(n, n, a["dx"], a["r0"], a["L0"], a["wt"], seed)
    layers = layers_of(cfg, seed, n)
    ctx.atm_set(layers, scr)
    return Workload(cfg=cfg, ctx=ctx, setup=setup, ipowfs=ip, wfs=wl, layers=layers, screens=scr)


@dataclass
class BatchWorkload:
    """Several WFS types (powfs) of one simulation on one device and one
    atmosphere: the uneven batch.  ``members`` holds (cfg, setup, ipowfs, wfs)."""
    ctx: "shwfs.Context"
    members: list
    layers: List[dict] = field(default_factory=list)
    screens: List[np.ndarray] = field(default_factory=list)
    graph: bool = True

    @property
    def nwfs(self) -> int:
        return sum(len(m[3]) for m in self.members)

    @property
    def images_per_frame(self) -> int:
        return sum(m[1].nsa * len(m[3]) for m in self.members)

    def frame(self, isim: int):
        """Queue one frame of every WFS of every member (as one CUDA graph when graph is set)."""
        if self.graph:
            self.ctx.frame_graph(isim, 0, self.nwfs)
        else:
            self.ctx.frame_queue(isim, 0, self.nwfs)

    def frame_sync(self, want_ints: bool = False, out=None):
        """Gradients of every WFS (with intensities when want_ints); without
        intensities, one wait and one copy for the whole frame, into ``out``
        when given (see Context.frame_sync_range)."""
        if not want_ints:
            return self.ctx.frame_sync_range(0, self.nwfs, out=out)
        out = []
        for _, _, ip, wl in self.members:
            out += [self.ctx.frame_sync(i, ip, want_ints) for i in wl]
        return out

    def close(self):
        self.ctx.close()
        for m in self.members:
            m[1].close()


def build_batch(cfgs, device: int = 0, seed: int = 1, noisy: bool = True, nx: int = None,
                form: int = shwfs.SHWFS_FORM_FFT, graph: bool = True) -> BatchWorkload:
    """One context holding every config of ``cfgs`` as its own powfs; the
    atmosphere (screens, winds, frame period) is that of the first config."""
    ctx = shwfs.Context(device)
    ctx.set_form(form)
    ctx.set_dt(cfgs[0].get("dt", 1.0 / 800))
    members = []
    nw = 0
    for j, cfg in enumerate(cfgs):
        setup = Setup(cfg)
        ip = setup.load(ctx)
        wl = []
        for k in range(cfg["nwfs"]):
            i = ctx.wfs_add(ipowfs=ip, thetax=cfg["thetax"][k], thetay=cfg["thetay"][k], hs=cfg["hs"], hc=0.0,
                            misregx=0.0, misregy=0.0, sigsim=cfg["siglev"], wvlwt=1.0, noisy=1 if noisy else 0)
            setup.load_wfs(ctx, i)
            ctx.wfs_seed(i, seed * 1000003 + nw)
            nw += 1
            wl.append(i)
        members.append((cfg, setup, ip, wl))
    a = cfgs[0]["atm"]
    n = nx or a["nx"]
    scr = screens(n, n, a["dx"], a["r0"], a["L0"], a["wt"], seed)
    layers = layers_of(cfgs[0], seed, n)
    ctx.atm_set(layers, scr)
    return BatchWorkload(ctx=ctx, members=members, layers=layers, screens=scr, graph=graph)
