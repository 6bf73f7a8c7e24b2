"""ctypes driver of the reference's own C code (oracle/_ref/libmaosref.so).

Test infrastructure.  The library is the reference's maos/, lib/, math/ and
sys/ sources compiled in place by ``make -C oracle ref`` with stand-ins for the
absent FFTW and BLAS/LAPACK (oracle/refbuild/).  :class:`RefPowfs` runs the
reference's SH setup (maos/powfs.c: setup_shwfs_geom, setup_shwfs_prep_phy,
setup_shwfs_dtf, setup_shwfs_etf, setup_powfs_llt, setup_shwfs_phygrad) and
exposes its outputs and per-frame routines (wfsints, shwfs_grad, addnoise,
prop).  The library holds one powfs at a time (global state, as in MAOS).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libmaosref.so")


class OrefCfg(C.Structure):
    _fields_ = [("D", C.c_double), ("Din", C.c_double), ("amp_binary", C.c_int), ("order", C.c_int),
                ("dsa", C.c_double), ("dx", C.c_double), ("saat", C.c_double), ("embfac", C.c_int),
                ("notf", C.c_int), ("pixpsa", C.c_int), ("pixtheta", C.c_double), ("pixblur", C.c_double),
                ("wvl", C.c_double), ("hs", C.c_double), ("siglev", C.c_double), ("rne", C.c_double),
                ("bkgrnd", C.c_double), ("bkgrndc", C.c_double), ("phytype", C.c_int), ("sigmatch", C.c_int),
                ("mtchcr", C.c_int), ("cogthres", C.c_double), ("cogoff", C.c_double), ("r0", C.c_double),
                ("L0", C.c_double), ("has_llt", C.c_int), ("llt_d", C.c_double), ("llt_widthp", C.c_double),
                ("llt_ox", C.c_double), ("llt_oy", C.c_double), ("na_n", C.c_int), ("na_h", C.c_void_p),
                ("na_p", C.c_void_p), ("nwfs", C.c_int), ("thetax", C.c_void_p), ("thetay", C.c_void_p),
                ("nthread", C.c_int), ("nwvl", C.c_int), ("wvls", C.c_void_p), ("wvlwts", C.c_void_p)]


_lib = None


def available() -> bool:
    return os.path.exists(REF_LIB)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{REF_LIB} is not built (make -C oracle ref)")
        L = C.CDLL(REF_LIB)
        for name in ("oref_nsa", "oref_nopd", "oref_notf", "oref_pixpsax", "oref_pixpsay", "oref_llt_nx", "oref_setup"):
            getattr(L, name).restype = C.c_int
        for name in ("oref_areascale", "oref_dtheta", "oref_get_ptsdx", "oref_get_i0sumsum", "oref_frame_mt",
                     "oref_frame_full_mt", "oref_get_saasum"):
            getattr(L, name).restype = C.c_double
        _lib = L
    return _lib


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class RefPowfs:
    """One powfs set up by the reference's own code from a config dict."""

    def __init__(self, cfg: dict, nthread: int = 1):
        self.cfg = cfg
        L = lib()
        keep = []
        na_h = na_p = None
        if cfg.get("has_llt"):
            from maos_b200.configs import sodium_gaussian
            s = cfg["sodium"]
            na_h, na_p = sodium_gaussian(s["centers"], s["fwhms"], s["weights"])
            keep += [na_h, na_p]
        tx = np.asarray(cfg["thetax"], dtype=np.float64)
        ty = np.asarray(cfg["thetay"], dtype=np.float64)
        keep += [tx, ty]
        # several wavelengths: cfg["wvls"] with weights cfg["wvlwts"] (powfs.wvl, powfs.wvlwts)
        wv = np.ascontiguousarray(cfg.get("wvls", [cfg["wvl"]]), dtype=np.float64)
        ww = np.ascontiguousarray(cfg.get("wvlwts", [1.0] * len(wv)), dtype=np.float64)
        keep += [wv, ww]
        c = OrefCfg(D=cfg["D"], Din=cfg["Din"], amp_binary=cfg.get("amp_binary", 0), order=cfg["order"],
                    dsa=cfg["dsa"], dx=cfg["dx"], saat=cfg["saat"], embfac=cfg["embfac"], notf=cfg["notf"],
                    pixpsa=cfg["pixpsa"], pixtheta=cfg["pixtheta"], pixblur=cfg["pixblur"], wvl=cfg["wvl"],
                    hs=cfg["hs"], siglev=cfg["siglev"], rne=cfg["rne"], bkgrnd=cfg.get("bkgrnd", 0.0),
                    bkgrndc=cfg.get("bkgrndc", 0.0), phytype=cfg["phytype"], sigmatch=cfg["sigmatch"],
                    mtchcr=cfg.get("mtchcr", 0), cogthres=cfg.get("cogthres", 0.0), cogoff=cfg.get("cogoff", 0.0),
                    r0=cfg["r0"], L0=cfg["L0"], has_llt=cfg.get("has_llt", 0), llt_d=cfg.get("llt_d", 0.0),
                    llt_widthp=cfg.get("llt_widthp", 0.0), llt_ox=cfg.get("llt_ox", 0.0),
                    llt_oy=cfg.get("llt_oy", 0.0), na_n=0 if na_h is None else len(na_h), na_h=_p(na_h),
                    na_p=_p(na_p), nwfs=cfg["nwfs"], thetax=_p(tx), thetay=_p(ty), nthread=nthread,
                    nwvl=len(wv), wvls=_p(wv), wvlwts=_p(ww))
        self._keep = keep
        self.nsa = L.oref_setup(C.byref(c))
        self.nopd = L.oref_nopd()
        self.notf = L.oref_notf()
        self.pixpsax = L.oref_pixpsax()
        self.pixpsay = L.oref_pixpsay()
        self.npix = self.pixpsax * self.pixpsay
        self.areascale = L.oref_areascale()
        self.dtheta = L.oref_dtheta()
        self.llt_nx = L.oref_llt_nx()

    # ---- setup outputs ----
    def saloc(self):
        x = np.zeros(self.nsa); y = np.zeros(self.nsa)
        lib().oref_get_saloc(_p(x), _p(y))
        return x, y

    def ptsorig(self):
        x = np.zeros(self.nsa); y = np.zeros(self.nsa)
        lib().oref_get_ptsorig(_p(x), _p(y))
        return x, y

    def ptsdx(self) -> float:
        return lib().oref_get_ptsdx()

    def amp(self):
        a = np.zeros(self.nsa * self.nopd ** 2)
        lib().oref_get_amp(_p(a))
        return a

    def saasum(self) -> float:
        return lib().oref_get_saasum()

    def saa(self):
        a = np.zeros(self.nsa)
        lib().oref_get_saa(_p(a))
        return a

    def select_wvl(self, iwvl: int):
        """The wavelength whose DTF nominal, pixel map, ETF and dtheta the getters return."""
        lib().oref_select_wvl(C.c_int(iwvl))
        self.dtheta = lib().oref_dtheta()

    def nominal(self, isa: int = 0):
        a = np.zeros(self.notf ** 2)
        lib().oref_get_nominal(C.c_int(isa), _p(a))
        return a

    def si_dense(self, isa: int = 0):
        a = np.zeros(self.npix * self.notf ** 2)
        lib().oref_get_si_dense(C.c_int(isa), _p(a))
        return a.reshape(self.notf ** 2, self.npix).T  # [pixel, psf index]

    def etf(self):
        n2 = self.notf ** 2
        out = np.zeros((self.nsa, n2), dtype=np.complex128)
        buf = np.zeros(2 * n2)
        for isa in range(self.nsa):
            lib().oref_get_etf(C.c_int(isa), _p(buf))
            out[isa] = buf[0::2] + 1j * buf[1::2]
        return out

    def setup_etf2(self, deltah: float, coldtrat: int):
        """Second ETF of the time interpolation (sodium focus at hs + deltah)
        and its period in frames."""
        lib().oref_setup_etf2(C.c_double(deltah), C.c_int(coldtrat))

    def etf2(self):
        n2 = self.notf ** 2
        out = np.zeros((self.nsa, n2), dtype=np.complex128)
        buf = np.zeros(2 * n2)
        for isa in range(self.nsa):
            lib().oref_get_etf2(C.c_int(isa), _p(buf))
            out[isa] = buf[0::2] + 1j * buf[1::2]
        return out

    def ztilt(self, opd):
        """Geometric z-tilt gradients (2 nsa) of an OPD (nsa nopd^2)."""
        g = np.zeros(2 * self.nsa)
        opd = np.ascontiguousarray(opd, dtype=np.float64)
        lib().oref_ztilt(_p(opd), _p(g))
        return g

    def gs0(self):
        """The G-tilt operator as MAOS CSC arrays: (nrow, ncol, pp, pi, px)."""
        L = lib()
        L.oref_gs0_nnz.restype = C.c_long
        nnz = L.oref_gs0_nnz()
        ncol = self.nsa * self.nopd ** 2
        pp = np.zeros(ncol + 1, dtype=np.int32)
        pi = np.zeros(nnz, dtype=np.int32)
        px = np.zeros(nnz)
        nr, nc = C.c_long(), C.c_long()
        L.oref_get_gs0(C.byref(nr), C.byref(nc), _p(pp), _p(pi), _p(px))
        assert nc.value == ncol
        return nr.value, nc.value, pp, pi, px

    def gtilt(self, opd):
        """G-tilt gradients GS0 opd (2 nsa)."""
        g = np.zeros(2 * self.nsa)
        opd = np.ascontiguousarray(opd, dtype=np.float64)
        lib().oref_gtilt(_p(opd), _p(g))
        return g

    def srot(self):
        a = np.zeros(self.nsa); lib().oref_get_srot(_p(a)); return a

    def srsa(self):
        a = np.zeros(self.nsa); lib().oref_get_srsa(_p(a)); return a

    def lltamp(self):
        a = np.zeros(self.llt_nx ** 2); lib().oref_get_lltamp(_p(a)); return a

    def mtche(self):
        out = np.zeros((self.nsa, 2 * self.npix))
        buf = np.zeros(2 * self.npix)
        for isa in range(self.nsa):
            lib().oref_get_mtche(C.c_int(isa), _p(buf))
            out[isa] = buf
        return out

    def sepsf(self, isa: int):
        n = self.notf
        a = np.zeros(n * n)
        lib().oref_get_sepsf(C.c_int(isa), _p(a))
        return a

    def i0(self, isa: int):
        """(i0, gx, gy) of subaperture isa, each npix."""
        i0, gx, gy = np.zeros(self.npix), np.zeros(self.npix), np.zeros(self.npix)
        lib().oref_get_i0(C.c_int(isa), _p(i0), _p(gx), _p(gy))
        return i0, gx, gy

    def i0sum(self):
        a = np.zeros(self.nsa); lib().oref_get_i0sum(_p(a)); return a

    def i0sumsum(self) -> float:
        return lib().oref_get_i0sumsum()

    # ---- per-frame routines ----
    def wfsints(self, opd, lltopd=None, iwfs=0, isa0=0, isa1=None, isim=0):
        ints = np.zeros(self.nsa * self.npix)
        opd = np.ascontiguousarray(opd, dtype=np.float64)
        llt = None if lltopd is None else np.ascontiguousarray(lltopd, dtype=np.float64)
        lib().oref_wfsints(C.c_int(iwfs), _p(opd), _p(llt), _p(ints), C.c_int(isa0),
                           C.c_int(self.nsa if isa1 is None else isa1), C.c_int(isim))
        return ints

    def grad(self, ints, iwfs=0):
        g = np.zeros(2 * self.nsa)
        ints = np.ascontiguousarray(ints, dtype=np.float64)
        lib().oref_shwfs_grad(C.c_int(iwfs), _p(ints), _p(g))
        return g

    def prop_layer(self, screen, dx, ox, oy, ht, thetax, thetay, hs, shiftx, shifty, opd=None, alpha=1.0, wrap=1):
        scr = np.ascontiguousarray(screen, dtype=np.float64)
        ny, nx = scr.shape
        if opd is None:
            opd = np.zeros(self.nsa * self.nopd ** 2)
        lib().oref_prop_layer(_p(scr), C.c_long(nx), C.c_long(ny), C.c_double(dx), C.c_double(ox), C.c_double(oy),
                              C.c_double(ht), C.c_double(thetax), C.c_double(thetay), C.c_double(hs),
                              C.c_double(shiftx), C.c_double(shifty), C.c_double(alpha), C.c_int(wrap), _p(opd),
                              C.c_int(0), C.c_int(self.nsa))
        return opd

    def prop_llt(self, screen, dx, ox, oy, ht, thetax, thetay, hs, shiftx, shifty, lltopd=None):
        scr = np.ascontiguousarray(screen, dtype=np.float64)
        ny, nx = scr.shape
        if lltopd is None:
            lltopd = np.zeros(self.llt_nx ** 2)
        lib().oref_prop_llt(_p(scr), C.c_long(nx), C.c_long(ny), C.c_double(dx), C.c_double(ox), C.c_double(oy),
                            C.c_double(ht), C.c_double(thetax), C.c_double(thetay), C.c_double(hs),
                            C.c_double(shiftx), C.c_double(shifty), _p(lltopd))
        return lltopd

    def frame_mt(self, opd, lltopd, seed=1, noisy=False, iwfs=0):
        ints = np.zeros(self.nsa * self.npix)
        g = np.zeros(2 * self.nsa)
        opd = np.ascontiguousarray(opd, dtype=np.float64)
        llt = None if lltopd is None else np.ascontiguousarray(lltopd, dtype=np.float64)
        t = lib().oref_frame_mt(C.c_int(iwfs), _p(opd), _p(llt), _p(ints), _p(g), C.c_uint(seed), C.c_int(int(noisy)))
        return ints, g, t


def atm_set(screens, layers):
    """Give the reference's full-frame path its turbulence (list of (ny,nx) screens,
    layer dicts with nx, ny, dx, ox, oy, ht, vx, vy)."""
    n = len(screens)
    keep = [np.ascontiguousarray(sc, dtype=np.float64) for sc in screens]
    ptrs = (C.c_void_p * n)(*[k.ctypes.data for k in keep])
    arr = lambda key, t=np.float64: np.ascontiguousarray([l[key] for l in layers], dtype=t)
    nx, ny = arr("nx", np.int64), arr("ny", np.int64)
    dx, ox, oy, ht, vx, vy = (arr(k) for k in ("dx", "ox", "oy", "ht", "vx", "vy"))
    lib().oref_atm_set(C.c_int(n), ptrs, _p(nx), _p(ny), _p(dx), _p(ox), _p(oy), _p(ht), _p(vx), _p(vy))


def cl_set(mirrors=(), surfaces=(), use_dm=False, ptt=(0.0, 0.0, 0.0), focus_tel=0.0, focus_llt=0.0,
           lltptt=(0.0, 0.0), opdadd=None):
    """Closed-loop terms of the full-frame path (mirror dicts: nx, ny, dx, ox, oy, ht)."""
    n = len(mirrors)
    keep = [np.ascontiguousarray(s, dtype=np.float64) for s in surfaces]
    ptrs = (C.c_void_p * max(n, 1))(*[k.ctypes.data for k in keep])
    arr = lambda key, t=np.float64: np.ascontiguousarray([m[key] for m in mirrors] or [0], dtype=t)
    nx, ny = arr("nx", np.int64), arr("ny", np.int64)
    dx, ox, oy, ht = (arr(k) for k in ("dx", "ox", "oy", "ht"))
    p = np.ascontiguousarray(ptt, dtype=np.float64)
    lp = np.ascontiguousarray(lltptt, dtype=np.float64)
    oa = None if opdadd is None else np.ascontiguousarray(opdadd, dtype=np.float64).ravel()
    lib().oref_cl_set(C.c_int(n), ptrs, _p(nx), _p(ny), _p(dx), _p(ox), _p(oy), _p(ht), C.c_int(int(bool(use_dm))),
                      _p(p), C.c_double(focus_tel), C.c_double(focus_llt), _p(lp), _p(oa))


def frame_opd(ref: "RefPowfs", iwfs: int, isim: int, dt: float):
    """(OPD, LLT OPD or None) of WFS iwfs at step isim on the full-frame path."""
    opd = np.zeros(ref.nsa * ref.nopd ** 2)
    llt = np.zeros(ref.llt_nx ** 2) if ref.llt_nx else None
    lib().oref_frame_opd(C.c_int(iwfs), C.c_int(isim), C.c_double(dt), _p(opd), _p(llt))
    return opd, llt


def frame_full_mt(ref: "RefPowfs", iwfs: int, isim: int, dt: float, seed: int = 1, noisy: bool = True):
    """One complete WFS frame of the reference CPU path; returns (ints, grad, seconds)."""
    ints = np.zeros(ref.nsa * ref.npix)
    g = np.zeros(2 * ref.nsa)
    t = lib().oref_frame_full_mt(C.c_int(iwfs), C.c_int(isim), C.c_double(dt), _p(ints), _p(g), C.c_uint(seed),
                                 C.c_int(int(noisy)))
    return ints, g, t


def si_to_taps(si_dense: np.ndarray):
    """Pixel sampling matrix (npix x notf^2) -> 4-tap (index, weight) arrays."""
    npix = si_dense.shape[0]
    idx = -np.ones((npix, 4), dtype=np.int32)
    wt = np.zeros((npix, 4))
    for p in range(npix):
        nz = np.nonzero(si_dense[p])[0]
        if len(nz) > 4:
            raise ValueError(f"pixel {p} has {len(nz)} taps")
        idx[p, :len(nz)] = nz
        wt[p, :len(nz)] = si_dense[p, nz]
    return idx, wt


def kat_psd() -> np.ndarray:
    out = np.zeros(7)
    lib().oref_kat_psd(_p(out))
    return out


def genatm_simple(r0, L0, slope, dx, n, seed):
    out = np.zeros(n * n)
    lib().oref_genatm_simple(C.c_double(r0), C.c_double(L0), C.c_double(slope), C.c_double(dx), C.c_long(n),
                             C.c_uint(seed), _p(out))
    return out.reshape(n, n)


def turbcov(r, r0, L0):
    """The reference's turbcov (rmax 0) at separations r."""
    r = np.ascontiguousarray(r, dtype=np.float64)
    out = np.zeros_like(r)
    lib().oref_turbcov(_p(r), C.c_long(r.size), C.c_double(r0), C.c_double(L0), _p(out))
    return out


def genscreen(nx, ny, dx, r0, L0, wt, seed):
    """Von Karman screens from the reference's genscreen: a list of (ny, nx) arrays, one per weight."""
    n = len(wt)
    outs = [np.zeros((ny, nx)) for _ in range(n)]
    ptrs = (C.c_void_p * n)(*[o.ctypes.data for o in outs])
    w = np.ascontiguousarray(wt, dtype=np.float64)
    lib().oref_genscreen(C.c_int(n), C.c_long(nx), C.c_long(ny), C.c_double(dx), C.c_double(r0), C.c_double(L0),
                         _p(w), C.c_uint(int(seed) & 0xFFFFFFFF), ptrs)
    return outs


class RefEvl:
    """The reference's science aperture and open-loop evaluation (setup_aper
    for an annulus; prop onto aper->locs, loc_calc_ptt, locfft_psf)."""

    def __init__(self, D, Din, dx, wvl=(), nembed=()):
        L = lib()
        L.oref_evl_setup.restype = C.c_long
        w = np.ascontiguousarray(wvl, dtype=np.float64)
        n = np.ascontiguousarray(nembed, dtype=np.int64)
        self.nwvl = len(w)
        self.nloc = L.oref_evl_setup(C.c_double(D), C.c_double(Din), C.c_double(dx), C.c_int(self.nwvl), _p(w), _p(n))
        self.dx = dx

    def aper(self):
        x, y, a = np.zeros(self.nloc), np.zeros(self.nloc), np.zeros(self.nloc)
        lib().oref_evl_get_aper(_p(x), _p(y), _p(a))
        return x, y, a

    def frame(self, thetax, thetay, hs, isim, dt, pttr=0, psfsize=None):
        """(opd, wfe[3], coeff[3], [psf per wavelength] or None)"""
        opd, wfe, coeff = np.zeros(self.nloc), np.zeros(3), np.zeros(3)
        psf = None
        ps = None
        if psfsize is not None:
            ps = np.ascontiguousarray(psfsize, dtype=np.int64)
            psf = np.zeros(int(np.sum(ps.astype(np.int64) ** 2)))
        lib().oref_evl_frame(C.c_double(thetax), C.c_double(thetay), C.c_double(hs), C.c_int(isim), C.c_double(dt),
                             C.c_int(pttr), C.c_int(self.nwvl), _p(ps), _p(opd), _p(wfe), _p(coeff), _p(psf))
        out = None
        if psf is not None:
            out, off = [], 0
            for n in ps:
                out.append(psf[off:off + n * n].reshape(n, n, order="F"))
                off += n * n
        return opd, wfe, coeff, out
