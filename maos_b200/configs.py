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

CONFIGS = {c["name"]: c for c in (NGS8, LGS30)}
