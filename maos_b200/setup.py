"""ctypes binding of the host setup producers (include/shwfs_setup.h).

:class:`Setup` builds a powfs from a configuration dict (maos_b200.configs):
subaperture geometry and valid mask, DTF nominal, pixel-sampling map, ETF and
LLT pupil for LGS, and the matched filter; :meth:`Setup.load` puts it into a
:class:`maos_b200.shwfs.Context`.  :func:`screens` makes von Karman phase
screens the way the reference does.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Sequence

import numpy as np

from . import shwfs
from .configs import sodium_gaussian

GET = dict(salocx=1, salocy=2, origx=3, origy=4, amp=5, saa=6, nominal=7, simap_wt=8, srot=9, srsa=10, etf=11,
           lltamp=12, mtche=13, i0sum=14, i0=15, gx=16, gy=17, sepsf=18, seotf=19)


class SetupCfg(C.Structure):
    _fields_ = [("D", C.c_double), ("Din", C.c_double), ("amp_binary", C.c_int), ("order", C.c_int),
                ("dsa", C.c_double), ("dx", C.c_double), ("saat", C.c_double), ("embfac", C.c_int),
                ("notf", C.c_int), ("pixpsa", C.c_int), ("pixtheta", C.c_double), ("pixblur", C.c_double),
                ("wvl", C.c_double), ("hs", C.c_double), ("siglev", C.c_double), ("rne", C.c_double),
                ("bkgrnd", C.c_double), ("bkgrndc", C.c_double), ("gradtype", C.c_int), ("sigmatch", C.c_int),
                ("mtchcr", C.c_int), ("cogthres", C.c_double), ("cogoff", C.c_double), ("has_llt", C.c_int),
                ("llt_d", C.c_double), ("llt_widthp", C.c_double), ("llt_ox", C.c_double), ("llt_oy", C.c_double),
                ("na_n", C.c_int), ("na_h", C.c_void_p), ("na_p", C.c_void_p), ("r0", C.c_double),
                ("L0", C.c_double)]


_bound = False


def _lib():
    global _bound
    L = shwfs.lib()
    if not _bound:
        vp, i, dp = C.c_void_p, C.c_int, C.POINTER(C.c_double)
        L.shwfs_setup_create.argtypes = [C.POINTER(vp), C.POINTER(SetupCfg)]
        L.shwfs_setup_destroy.argtypes = [vp]
        L.shwfs_setup_destroy.restype = None
        L.shwfs_setup_error.argtypes = [vp]
        L.shwfs_setup_error.restype = C.c_char_p
        for n in ("nsa", "nopd", "notf", "npix", "llt_nx"):
            f = getattr(L, f"shwfs_setup_{n}")
            f.argtypes = [vp]
            f.restype = i
        for n in ("dx", "areascale", "dtheta", "i0sumsum", "saasum"):
            f = getattr(L, f"shwfs_setup_{n}")
            f.argtypes = [vp]
            f.restype = C.c_double
        L.shwfs_setup_get.argtypes = [vp, i, dp]
        L.shwfs_setup_get_simap_idx.argtypes = [vp, C.POINTER(C.c_int)]
        L.shwfs_setup_load.argtypes = [vp, vp, C.POINTER(i)]
        L.shwfs_setup_load_wfs.argtypes = [vp, vp, i]
        L.shwfs_setup_load_band.argtypes = [vp, vp, i, C.c_double, C.POINTER(i)]
        L.shwfs_screens_vonkarman.argtypes = [C.POINTER(dp), i, C.c_long, C.c_long, C.c_double, C.c_double, C.c_double,
                                             dp, C.c_uint32]
        L.shwfs_aper_build.argtypes = [C.c_double, C.c_double, C.c_double, C.POINTER(C.c_long), dp, dp, dp]
        L.shwfs_aper_build.restype = i
        _bound = True
    return L


class Setup:
    """Setup of one powfs, built by the native host code from a config dict."""

    def __init__(self, cfg: dict):
        L = _lib()
        self.cfg = cfg
        self._keep = []
        na_h = na_p = None
        if cfg.get("has_llt"):
            s = cfg["sodium"]
            na_h, na_p = sodium_gaussian(s["centers"], s["fwhms"], s["weights"])
            self._keep += [na_h, na_p]
        c = SetupCfg(D=cfg["D"], Din=cfg["Din"], amp_binary=cfg.get("amp_binary", 0), order=cfg["order"],
                     dsa=cfg["dsa"], dx=cfg["dx"], saat=cfg["saat"], embfac=cfg["embfac"], notf=cfg["notf"],
                     pixpsa=cfg["pixpsa"], pixtheta=cfg["pixtheta"], pixblur=cfg["pixblur"], wvl=cfg["wvl"],
                     hs=cfg["hs"], siglev=cfg["siglev"], rne=cfg["rne"], bkgrnd=cfg.get("bkgrnd", 0.0),
                     bkgrndc=cfg.get("bkgrndc", 0.0), gradtype=cfg["phytype"], sigmatch=cfg["sigmatch"],
                     mtchcr=cfg.get("mtchcr", 0), cogthres=cfg.get("cogthres", 0.0), cogoff=cfg.get("cogoff", 0.0),
                     has_llt=cfg.get("has_llt", 0), llt_d=cfg.get("llt_d", 0.0), llt_widthp=cfg.get("llt_widthp", 0.0),
                     llt_ox=cfg.get("llt_ox", 0.0), llt_oy=cfg.get("llt_oy", 0.0),
                     na_n=0 if na_h is None else len(na_h),
                     na_h=None if na_h is None else na_h.ctypes.data, na_p=None if na_p is None else na_p.ctypes.data,
                     r0=cfg.get("r0", 0.0), L0=cfg.get("L0", math.inf))
        h = C.c_void_p()
        rc = L.shwfs_setup_create(C.byref(h), C.byref(c))
        self._h = h
        if rc != 0:
            msg = L.shwfs_setup_error(h).decode() if h else str(rc)
            self.close()
            raise shwfs.ShwfsError(f"setup: {msg}")
        self.nsa = L.shwfs_setup_nsa(h)
        self.nopd = L.shwfs_setup_nopd(h)
        self.notf = L.shwfs_setup_notf(h)
        self.npix = L.shwfs_setup_npix(h)
        self.llt_nx = L.shwfs_setup_llt_nx(h)
        self.dx = L.shwfs_setup_dx(h)
        self.areascale = L.shwfs_setup_areascale(h)
        self.dtheta = L.shwfs_setup_dtheta(h)
        self.i0sumsum = L.shwfs_setup_i0sumsum(h)
        self.saasum = L.shwfs_setup_saasum(h)

    def close(self):
        if getattr(self, "_h", None):
            _lib().shwfs_setup_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _size(self, name):
        nsa, n2, np_, no2 = self.nsa, self.notf ** 2, self.npix, self.nopd ** 2
        return dict(salocx=nsa, salocy=nsa, origx=nsa, origy=nsa, amp=nsa * no2, saa=nsa, nominal=n2,
                    simap_wt=np_ * 4, srot=nsa, srsa=nsa, etf=2 * nsa * n2, lltamp=self.llt_nx ** 2,
                    mtche=nsa * 2 * np_, i0sum=nsa, i0=nsa * np_, gx=nsa * np_, gy=nsa * np_, sepsf=nsa * n2,
                    seotf=2 * nsa * n2)[name]

    def get(self, name: str) -> np.ndarray:
        out = np.zeros(self._size(name))
        rc = _lib().shwfs_setup_get(self._h, GET[name], out.ctypes.data_as(C.POINTER(C.c_double)))
        if rc != 0:
            raise shwfs.ShwfsError(f"setup array {name} is not available")
        if name in ("etf", "seotf"):
            return (out[0::2] + 1j * out[1::2]).reshape(self.nsa, self.notf ** 2)
        return out

    def simap_idx(self) -> np.ndarray:
        out = np.zeros(self.npix * 4, dtype=np.int32)
        rc = _lib().shwfs_setup_get_simap_idx(self._h, out.ctypes.data_as(C.POINTER(C.c_int)))
        if rc != 0:
            raise shwfs.ShwfsError("pixel map is not available")
        return out

    def load(self, ctx: "shwfs.Context") -> int:
        ip = C.c_int()
        ctx._check(_lib().shwfs_setup_load(self._h, ctx._h, C.byref(ip)), "setup_load")
        ctx.npix[ip.value] = self.npix
        ctx.nsa[ip.value] = self.nsa
        return ip.value

    def load_band(self, ctx: "shwfs.Context", ipowfs: int, wvlwt: float) -> int:
        """This setup as a further wavelength band of powfs ipowfs (weight wvlwt);
        returns the band's powfs index."""
        ib = C.c_int()
        ctx._check(_lib().shwfs_setup_load_band(self._h, ctx._h, ipowfs, float(wvlwt), C.byref(ib)), "setup_load_band")
        ctx.npix[ib.value] = self.npix
        ctx.nsa[ib.value] = self.nsa
        return ib.value

    def load_wfs(self, ctx: "shwfs.Context", iwfs: int):
        ctx._check(_lib().shwfs_setup_load_wfs(self._h, ctx._h, iwfs), "setup_load_wfs")


def screens(nx: int, ny: int, dx: float, r0: float, L0: float, wt: Sequence[float], seed: int):
    """Von Karman screens (nlayer = len(wt)) as a list of (ny, nx) float64 arrays."""
    L = _lib()
    n = len(wt)
    outs = [np.zeros((ny, nx)) for _ in range(n)]
    ptrs = (C.POINTER(C.c_double) * n)(*[o.ctypes.data_as(C.POINTER(C.c_double)) for o in outs])
    w = np.ascontiguousarray(wt, dtype=np.float64)
    rc = L.shwfs_screens_vonkarman(ptrs, n, nx, ny, dx, r0, L0, w.ctypes.data_as(C.POINTER(C.c_double)),
                                   int(seed) & 0xFFFFFFFF)
    if rc != 0:
        raise shwfs.ShwfsError("screen generation failed")
    return outs


def aperture(D: float, Din: float, dx: float):
    """Science aperture of an annulus sampled at dx (shwfs_aper_build): (locx,
    locy, amp) with the amplitude normalised to sum 1."""
    L = _lib()
    n = C.c_long()
    if L.shwfs_aper_build(D, Din, dx, C.byref(n), None, None, None) != 0:
        raise shwfs.ShwfsError("aperture: bad arguments")
    x, y, a = np.zeros(n.value), np.zeros(n.value), np.zeros(n.value)
    dp = C.POINTER(C.c_double)
    if L.shwfs_aper_build(D, Din, dx, C.byref(n), x.ctypes.data_as(dp), y.ctypes.data_as(dp), a.ctypes.data_as(dp)):
        raise shwfs.ShwfsError("aperture: build failed")
    return x, y, a
