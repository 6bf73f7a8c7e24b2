"""Workload definitions for the Shack-Hartmann frame.

Each configuration names the telescope, atmosphere and WFS parameters of one
benchmark case, in the reference's parameter vocabulary (powfs.*, wfs.*,
atm.*, llt.*).  Angles are stored in radians.
"""
from __future__ import annotations

import math

AS2RAD = 4.848136811095360e-06  # arcsec in radian (lib/libmisc.c:23)


def _lgs_dirs(n: int, radius_as: float):
    return ([radius_as * AS2RAD * math.cos(2 * math.pi * k / n) for k in range(n)],
            [radius_as * AS2RAD * math.sin(2 * math.pi * k / n) for k in range(n)])


def sodium_gaussian(centers_m, fwhms_m, weights, hmin=80e3, hmax=100e3, n=201):
    """Evenly sampled sodium profile (altitude, strength) summing to 1."""
    import numpy as np
    h = np.linspace(hmin, hmax, n)
    p = np.zeros_like(h)
    for c, f, w in zip(centers_m, fwhms_m, weights):
        s = f / (2 * math.sqrt(2 * math.log(2)))
        p += w * np.exp(-0.5 * ((h - c) / s) ** 2)
    p /= p.sum()
    return h, p


# NGS, 8 m telescope, 16x16 subapertures, CoG.
NGS8 = dict(
    name="ngs8_16x16_cog",
    D=8.0, Din=1.2, amp_binary=1,
    order=16, dsa=0.5, dx=1.0 / 32, saat=0.3, embfac=2, notf=32,
    pixpsa=8, pixtheta=0.5 * AS2RAD, pixblur=0.3, wvl=0.7e-6, hs=math.inf,
    siglev=1000.0, rne=3.0, bkgrnd=0.0, bkgrndc=0.0,
    phytype=2, sigmatch=1, mtchcr=0, cogthres=0.0, cogoff=0.0,
    r0=0.186, L0=30.0,
    has_llt=0, nwfs=1, thetax=[0.0], thetay=[0.0],
    atm=dict(r0=0.186, L0=30.0, nx=2048, dx=1.0 / 32, ht=[0.0, 10e3], wt=[0.7, 0.3],
             ws=[8.0, 20.0], wdir_deg=[0.0, 90.0]),
    dt=1.0 / 800,
)

_tx, _ty = _lgs_dirs(6, 35.0)
# NFIRAOS-like: 30 m, 6 LGS at 35", 60x60 subapertures, matched filter.
LGS30 = dict(
    name="lgs30_6x60x60_mf",
    D=30.0, Din=3.6, amp_binary=0,
    order=60, dsa=0.5, dx=1.0 / 32, saat=0.3, embfac=2, notf=32,
    pixpsa=6, pixtheta=1.0 * AS2RAD, pixblur=0.3, wvl=0.589e-6, hs=90e3,
    siglev=500.0, rne=3.0, bkgrnd=0.0, bkgrndc=0.0,
    phytype=1, sigmatch=1, mtchcr=1, cogthres=0.0, cogoff=0.0,
    r0=0.186, L0=30.0,
    has_llt=1, llt_d=0.4, llt_widthp=0.6, llt_ox=8.0, llt_oy=0.0,
    sodium=dict(centers=[90e3], fwhms=[10e3], weights=[1.0]),
    nwfs=6, thetax=_tx, thetay=_ty,
    atm=dict(r0=0.186, L0=30.0, nx=2048, dx=1.0 / 32,
             ht=[0.0, 500.0, 1e3, 2e3, 4e3, 8e3, 16e3],
             wt=[0.596, 0.0386, 0.0386, 0.0386, 0.1436, 0.0386, 0.1024],
             ws=[5.6, 5.8, 6.3, 7.6, 13.3, 15.0, 12.1], wdir_deg=None),
    dt=1.0 / 800,
)

# Large-sampling stress: the LGS sensors of LGS30 sampled at 1/64 m (32x32 OPD
# points per subaperture), FFT 64, 12x12 pixels of 0.8", a two-Gaussian sodium
# layer at 88 and 94 km, screens of 4096^2 at 1/64 m.
LGS30_N64 = dict(
    LGS30, name="lgs30_6x60x60_n64",
    dx=1.0 / 64, notf=64, pixpsa=12, pixtheta=0.8 * AS2RAD,
    sodium=dict(centers=[88e3, 94e3], fwhms=[5e3, 5e3], weights=[0.6, 0.4]),
    atm=dict(LGS30["atm"], nx=4096, dx=1.0 / 64),
)

# Uneven batch members beside the LGS30 sensors: one NGS of 2x2 subapertures
# (64x64 OPD points each, FFT 128, 16x16 pixels of 4 mas) and two tip-tilt
# NGS of 1x1 (128x128 points, FFT 256), both at 1.65 um, CoG gradients.
NGS30_2X2 = dict(
    name="ngs30_2x2_n128",
    D=30.0, Din=3.6, amp_binary=0,
    order=2, dsa=15.0, dx=15.0 / 64, saat=0.3, embfac=2, notf=128,
    pixpsa=16, pixtheta=0.004 * AS2RAD, pixblur=0.3, wvl=1.65e-6, hs=math.inf,
    siglev=1000.0, rne=3.0, bkgrnd=0.0, bkgrndc=0.0,
    phytype=2, sigmatch=1, mtchcr=0, cogthres=0.0, cogoff=0.0,
    r0=0.186, L0=30.0,
    has_llt=0, nwfs=1, thetax=[0.0], thetay=[0.0],
    atm=LGS30["atm"], dt=1.0 / 800,
)
TT30 = dict(
    NGS30_2X2, name="tt30_1x1_n256",
    order=1, dsa=30.0, dx=30.0 / 128, notf=256,
    nwfs=2, thetax=[30.0 * AS2RAD, -30.0 * AS2RAD], thetay=[0.0, 0.0],
)

# Reduced copies for parity tests (the reference's CPU frame in seconds): an
# 8 m telescope with 8x8 LGS subapertures at the stress sampling.
LGS8_N64 = dict(
    LGS30_N64, name="lgs8_2x8x8_n64",
    D=4.0, Din=0.5, order=8, llt_ox=2.0, nwfs=2, thetax=[10.0 * AS2RAD, -10.0 * AS2RAD], thetay=[0.0, 5.0 * AS2RAD],
    atm=dict(LGS30["atm"], nx=512, dx=1.0 / 64),
)

# The LGS30 sensor (16x16 OPD points, FFT 32, 6x6 pixels, matched filter) on
# an 8 m telescope with 16x16 subapertures: a parity-test case small enough
# for committed fixtures.
LGS8_N32 = dict(
    LGS30, name="lgs8_2x16x16_mf",
    D=8.0, Din=1.2, order=16, llt_ox=4.0, nwfs=2, thetax=[10.0 * AS2RAD, -10.0 * AS2RAD], thetay=[0.0, 5.0 * AS2RAD],
    atm=dict(LGS30["atm"], nx=512),
)

# Polychromatic sensors (powfs.wvl with weights powfs.wvlwts): the NGS at 0.7
# and 0.9 um, the 8 m LGS at 0.589 and 0.62 um; the first wavelength is the
# one the OTF size and the main band use.
NGS8_2WVL = dict(NGS8, name="ngs8_16x16_2wvl", wvls=[0.7e-6, 0.9e-6], wvlwts=[0.6, 0.4])
LGS8_N32_2WVL = dict(LGS8_N32, name="lgs8_2x16x16_mf_2wvl", wvls=[0.589e-6, 0.62e-6], wvlwts=[0.7, 0.3])
LGS8_N64_2WVL = dict(LGS8_N64, name="lgs8_2x8x8_n64_2wvl", wvls=[0.589e-6, 0.62e-6], wvlwts=[0.7, 0.3])

CONFIGS = {c["name"]: c for c in (NGS8, LGS30, LGS30_N64, NGS30_2X2, TT30, LGS8_N64, LGS8_N32, NGS8_2WVL,
                                  LGS8_N32_2WVL, LGS8_N64_2WVL)}

# Science path: the 30 m aperture sampled at 1/64 m (the reference's default
# evl.dx = atm.dx), 9 directions on a 3x3 grid over a 30" field, PSFs at J, H
# and K (evl.wvl) on a 4096-point grid cropped to 1024 pixels, on the
# 7-layer atmosphere of the stress configuration (4096^2 screens at 1/64 m).
SCIENCE30 = dict(
    name="science_30m_9dir",
    D=30.0, Din=3.6, dx=1.0 / 64,
    dirs=[(x * AS2RAD, y * AS2RAD, math.inf) for y in (-15.0, 0.0, 15.0) for x in (-15.0, 0.0, 15.0)],
    wvl=[1.25e-6, 1.65e-6, 2.2e-6], nembed=[4096, 4096, 4096], psfsize=[1024, 1024, 1024], pttr=0,
    atm=LGS30_N64["atm"], dt=1.0 / 800,
)
SCIENCE = {SCIENCE30["name"]: SCIENCE30}

# The uneven batch: six LGS of LGS30 (FFT 32), the 2x2 NGS (FFT 128) and the
# two tip-tilt sensors (FFT 256) in one frame, on the LGS30 atmosphere.
UNEVEN_BATCH = dict(name="uneven_batch_lgs6_ngs1_tt2", members=[LGS30, NGS30_2X2, TT30])
BATCHES = {UNEVEN_BATCH["name"]: UNEVEN_BATCH}


def wind(cfg: dict, seed: int):
    """Per-layer wind vectors (vx, vy): speeds from the config, directions
    from a seeded generator unless the config fixes them."""
    import numpy as np
    a = cfg["atm"]
    rng = np.random.default_rng(seed)
    nl = len(a["ht"])
    if a.get("wdir_deg") is not None:
        ang = np.deg2rad(np.asarray(a["wdir_deg"], dtype=float))
    else:
        ang = rng.uniform(0, 2 * math.pi, nl)
    ws = np.asarray(a["ws"], dtype=float)
    return ws * np.cos(ang), ws * np.sin(ang)


def layers_of(cfg: dict, seed: int, nx: int = None):
    """Layer descriptors (screen size and origin, height, wind) of a config's
    atmosphere on nx x nx screens centred on the telescope."""
    a = cfg["atm"]
    n = nx or a["nx"]
    dx = a["dx"]
    vx, vy = wind(cfg, seed)
    o = -n / 2 * dx
    return [dict(nx=n, ny=n, dx=dx, ox=o, oy=o, ht=float(h), vx=float(vx[i]), vy=float(vy[i]), alpha=1.0)
            for i, h in enumerate(a["ht"])]


def workload_desc(cfg: dict, nsa: int, notf: int, npix: int) -> dict:
    """The workload of one frame of a config, as both bench arms name it."""
    a = cfg["atm"]
    return {"workload": cfg["name"], "wfs": cfg["nwfs"], "subapertures_per_wfs": nsa, "fft": notf,
            "pixels": npix, "layers": len(a["ht"]), "screen": f"{a['nx']}^2",
            "photons": cfg["siglev"], "read_noise_e": cfg["rne"],
            "gradients": "matched filter" if cfg["phytype"] == 1 else "CoG",
            "step": f"one frame of all {cfg['nwfs']} WFS: ray trace, uplink, imaging, noise, gradients"}

