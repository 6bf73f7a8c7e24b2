"""Writes the golden fixtures of tests/golden/ from the reference's own code.

Every number in the fixtures comes from the reference's C sources compiled in
place (oracle/_ref/libmaosref.so, ``make -C oracle ref``), and every file is
written by the reference's own .bin writer (writebin, math/cell.c:330-337):

- the OPD of one WFS by its ray tracer (prop_range, lib/accphi.c) on
  von Karman screens from its screen generator (lib/turbulence.c), with the
  same screens, winds and frame index as the GPU tests; stored in FP32, the
  precision the GPU path reads, and handed to the reference as those FP32
  values promoted to FP64;
- the LGS uplink OPD (prop of the LLT pupil);
- noise-free intensities (wfsints, maos/wfsints.c) and gradients (shwfs_grad,
  maos/utils.c) of that OPD;
- for matched-filter sensors the reference's matched filter (mtch,
  lib/mtch.c: a cell of nsa members of 2 x npix) and i0sum (i0sumsum in the
  header);
- geometric z-tilt (pts_ztilt, math/loc.c) and G-tilt gradients (GS0 opd,
  GS0 from mkg, lib/mkg.c) of the NGS OPD, and GS0 itself (gzip stream);
- the science path of a 4 m annulus (setup_aper, maos/aper.c): the OPD of
  two directions on aper->locs, their PR/TT/PTTR and piston/tip/tilt
  (loc_calc_ptt, math/loc.c) and PSF (locfft_psf, lib/locfft.c, |.|^2).

Needs the reference tree (it builds the oracle); the fixtures it writes
travel with the repository.  Run from the repository root:
``python tests/golden/make_golden.py``.
"""
from __future__ import annotations

import ctypes as C
import gzip
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from maos_b200.configs import NGS8, LGS8_N32, LGS8_N64  # noqa: E402
from maos_b200.setup import screens  # noqa: E402
from maos_b200.workload import wind  # noqa: E402
from oracle import ref  # noqa: E402

# (case name, config, WFS index, frame index, screen size, screen seed)
CASES = [
    ("ngs8", NGS8, 0, 5, 512, 11),
    ("lgs8_n32", LGS8_N32, 1, 7, 512, 12),
    ("lgs8_n64", LGS8_N64, 0, 3, 512, 13),
]


def layers_of(cfg, nx, seed):
    a = cfg["atm"]
    scr = screens(nx, nx, a["dx"], a["r0"], a["L0"], a["wt"], seed)
    vx, vy = wind(cfg, seed)
    o = -nx / 2 * a["dx"]
    lay = [dict(nx=nx, ny=nx, dx=a["dx"], ox=o, oy=o, ht=float(h), vx=float(vx[i]), vy=float(vy[i]))
           for i, h in enumerate(a["ht"])]
    return scr, lay


def trace(r, cfg, iwfs, isim, scr, lay):
    """OPD and (LGS) LLT OPD of one WFS at frame isim, by the reference's
    ray tracer, as its frame does (maos/wfsgrad.c:187-189, 337-365)."""
    dt = cfg["dt"]
    tx, ty, hs = cfg["thetax"][iwfs], cfg["thetay"][iwfs], cfg["hs"]
    opd = np.zeros(r.nsa * r.nopd ** 2)
    for L, s in zip(lay, scr):
        r.prop_layer(s, L["dx"], L["ox"], L["oy"], L["ht"], tx, ty, hs, -L["vx"] * dt * isim, -L["vy"] * dt * isim,
                     opd=opd)
    llt = None
    if cfg.get("has_llt"):
        ox, oy = cfg["llt_ox"], cfg.get("llt_oy", 0.0)
        llt = np.zeros(r.llt_nx ** 2)
        for L, s in zip(lay, scr):
            if 1.0 - L["ht"] / hs < 0:
                continue
            r.prop_llt(s, L["dx"], L["ox"], L["oy"], L["ht"], tx - ox / hs, ty - oy / hs, hs,
                       ox - L["vx"] * isim * dt, oy - L["vy"] * isim * dt, lltopd=llt)
    return opd, llt


def write_d(L, fn, a, nx, ny, kw=None):
    a = np.asfortranarray(np.asarray(a, dtype=np.float64).reshape(nx, ny, order="F"))
    L.oref_writebin_d(fn.encode(), a.ctypes.data_as(C.c_void_p), C.c_long(nx), C.c_long(ny),
                      kw.encode() if kw else None)


def write_f(L, fn, a, kw=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    L.oref_writebin_f(fn.encode(), a.ctypes.data_as(C.c_void_p), C.c_long(a.size), C.c_long(1),
                      kw.encode() if kw else None)


# Science path: aperture (D, Din, dx), PSF (wavelength, grid, crop), pttr,
# directions (thetax, thetay, hs), frame index, screen size and seed.
EVL_CASE = dict(name="evl4", D=4.0, Din=0.5, dx=1.0 / 16, wvl=[1.65e-6], nembed=[256], psfsize=[64], pttr=1,
                dirs=[(0.0, 0.0, math.inf), (10.0 * math.pi / 648000, -5.0 * math.pi / 648000, 90e3)],
                isim=9, nx=512, seed=14, cfg=LGS8_N32)


def write_evl(L):
    c = EVL_CASE
    scr, lay = layers_of(c["cfg"], c["nx"], c["seed"])
    ref.atm_set(scr, lay)
    e = ref.RefEvl(c["D"], c["Din"], c["dx"], wvl=c["wvl"], nembed=c["nembed"])
    kw = (f"D={c['D']}\nDin={c['Din']}\ndx={c['dx']!r}\nwvl={c['wvl'][0]!r}\nnembed={c['nembed'][0]}\n"
          f"psfsize={c['psfsize'][0]}\npttr={c['pttr']}\nisim={c['isim']}\nscreen_config={c['cfg']['name']}\n"
          f"screen_nx={c['nx']}\nscreen_seed={c['seed']}\nndir={len(c['dirs'])}")
    for k, (tx, ty, hs) in enumerate(c["dirs"]):
        opd, wfe, coeff, psf = e.frame(tx, ty, hs, c["isim"], c["cfg"]["dt"], pttr=c["pttr"], psfsize=c["psfsize"])
        p = lambda what: os.path.join(HERE, f"{c['name']}_dir{k}_{what}.bin")  # noqa: E731
        write_d(L, p("opd"), opd, len(opd), 1, kw=kw + f"\nthetax={tx!r}\nthetay={ty!r}\nhs={hs!r}")
        write_d(L, p("wfe"), np.concatenate([wfe, coeff]), 6, 1)
        write_d(L, p("psf"), psf[0].ravel(order="F"), c["psfsize"][0], c["psfsize"][0])
    print(c["name"], "nloc", e.nloc)


def main():
    L = ref.lib()
    write_evl(L)
    for name, cfg, iwfs, isim, nx, seed in CASES:
        r = ref.RefPowfs(cfg)
        scr, lay = layers_of(cfg, nx, seed)
        opd, llt = trace(r, cfg, iwfs, isim, scr, lay)
        opd32 = opd.astype(np.float32)
        llt32 = llt.astype(np.float32) if llt is not None else None
        kw = f"config={cfg['name']}\niwfs={iwfs}\nisim={isim}\nscreen_nx={nx}\nscreen_seed={seed}"
        p = lambda what: os.path.join(HERE, f"{name}_{what}.bin")  # noqa: E731
        write_f(L, p("opd"), opd32, kw)
        if llt32 is not None:
            write_f(L, p("lltopd"), llt32, kw)
        ints = r.wfsints(opd32.astype(np.float64), None if llt32 is None else llt32.astype(np.float64), iwfs=iwfs,
                         isim=isim)
        grad = r.grad(ints, iwfs=iwfs)
        write_d(L, p("ints"), ints, r.npix, r.nsa)
        write_d(L, p("grad"), grad, 2 * r.nsa, 1)
        if cfg["phytype"] == 1:
            m = r.mtche()
            n = r.nsa
            nxs = (C.c_long * n)(*([2 * r.npix] * n))
            nys = (C.c_long * n)(*([1] * n))
            keep = [np.ascontiguousarray(m[i]) for i in range(n)]
            ptrs = (C.c_void_p * n)(*[k.ctypes.data for k in keep])
            L.oref_writebin_dcell(p("mtche").encode(), n, nxs, nys, ptrs, None)
            write_d(L, p("i0sum"), r.i0sum(), r.nsa, 1, kw=f"i0sumsum={r.i0sumsum()!r}")
        if not cfg.get("has_llt"):
            o64 = opd32.astype(np.float64)
            write_d(L, p("ztilt"), r.ztilt(o64), 2 * r.nsa, 1)
            write_d(L, p("gtilt"), r.gtilt(o64), 2 * r.nsa, 1)
            # GS0 is large and sparse: the reference's file, gzip-compressed
            L.oref_writebin_gs0(p("gs0").encode())
            with open(p("gs0"), "rb") as f, open(p("gs0") + ".gz", "wb") as g:
                g.write(gzip.compress(f.read(), compresslevel=9, mtime=0))
            os.remove(p("gs0"))
        print(name, "nsa", r.nsa, "npix", r.npix, "max |g|", float(np.abs(grad).max()))


if __name__ == "__main__":
    main()
