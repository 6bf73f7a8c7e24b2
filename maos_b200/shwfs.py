"""ctypes binding of the C ABI declared in include/shwfs_b200.h.

This is the host-side mirror of the reference's GPU WFS seam
(cuda/sim/gpu_sim.h:39-48): a :class:`Context` holds the static data of the
powfs/WFS (what gpu_wfsgrad_init uploads), the turbulence screens (what
gpu_atm2gpu uploads) and runs frames (gpu_wfsgrad_queue/sync).  Errors are
raised as :class:`ShwfsError`, mirroring the reference's ``error()`` abort.

There is no CPU fallback: if the native library is missing the import of this
module fails.
"""
from __future__ import annotations

import atexit
import ctypes as C
import math
import os
import weakref
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libshwfs_b200.so")

SHWFS_GRAD_MF = 1
SHWFS_GRAD_COG = 2
SHWFS_GRAD_ZTILT = 3
SHWFS_GRAD_GTILT = 4
SHWFS_FORM_FFT = 0
SHWFS_FORM_TC = 1
SHWFS_TRACE_AUTO = 0
SHWFS_TRACE_LISTED = 1
SHWFS_TRACE_INTERLEAVED = 2


class ShwfsError(RuntimeError):
    pass


class PowfsDesc(C.Structure):
    _fields_ = [
        ("nsa", C.c_int), ("nopd", C.c_int), ("embfac", C.c_int), ("notf", C.c_int),
        ("pixpsax", C.c_int), ("pixpsay", C.c_int),
        ("pixthetax", C.c_double), ("pixthetay", C.c_double),
        ("wvl", C.c_double), ("dsa", C.c_double), ("dx", C.c_double), ("areascale", C.c_double),
        ("hs", C.c_double),
        ("has_etf", C.c_int), ("has_llt", C.c_int), ("llt_nx", C.c_int),
        ("llt_ox", C.c_double), ("llt_oy", C.c_double), ("llt_origx", C.c_double), ("llt_origy", C.c_double),
        ("gradtype", C.c_int), ("sigmatch", C.c_int),
        ("cogthres", C.c_double), ("cogoff", C.c_double),
        ("rne", C.c_double), ("bkgrnd", C.c_double), ("bkgrndc", C.c_double),
        ("saat", C.c_double), ("sigtot_cog", C.c_double),
    ]


class WfsDesc(C.Structure):
    _fields_ = [
        ("ipowfs", C.c_int),
        ("thetax", C.c_double), ("thetay", C.c_double),
        ("hs", C.c_double), ("hc", C.c_double),
        ("misregx", C.c_double), ("misregy", C.c_double),
        ("sigsim", C.c_double), ("wvlwt", C.c_double),
        ("noisy", C.c_int),
    ]


class LayerDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_long), ("ny", C.c_long),
        ("dx", C.c_double), ("ox", C.c_double), ("oy", C.c_double),
        ("ht", C.c_double), ("vx", C.c_double), ("vy", C.c_double),
        ("alpha", C.c_double),
    ]


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"native library {LIB_PATH} is missing; build it with `python -m maos_b200.build`")
    lib = C.CDLL(LIB_PATH)
    vp, ip, dp, i = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int
    sig = {
        "shwfs_create": [C.POINTER(vp), i],
        "shwfs_destroy": [vp],
        "shwfs_powfs_add": [vp, C.POINTER(PowfsDesc), ip],
        "shwfs_powfs_set_geom": [vp, i, dp, dp, dp, i, dp],
        "shwfs_powfs_set_nominal": [vp, i, dp, i],
        "shwfs_powfs_set_simap": [vp, i, ip, dp, i],
        "shwfs_powfs_set_etf": [vp, i, dp, i],
        "shwfs_powfs_set_lltamp": [vp, i, dp],
        "shwfs_wfs_add": [vp, C.POINTER(WfsDesc), ip],
        "shwfs_wfs_set_mtche": [vp, i, dp, dp, C.c_double],
        "shwfs_wfs_seed": [vp, i, C.c_uint64],
        "shwfs_atm_set": [vp, i, C.POINTER(LayerDesc), C.POINTER(dp)],
        "shwfs_set_form": [vp, i],
        "shwfs_set_dt": [vp, C.c_double],
        "shwfs_frame_queue": [vp, i, i, i],
        "shwfs_frame_sync": [vp, i, dp, dp],
        "shwfs_raytrace_dev": [vp, i, i, vp],
        "shwfs_ints_grad_dev": [vp, i, i, vp, vp, vp, vp, i],
        "shwfs_grad_dev": [vp, i, vp, vp],
        "shwfs_frame_graph": [vp, i, i, i],
        "shwfs_wfs_update_mtche": [vp, i, i],
        "shwfs_frame_sync_range": [vp, i, i, dp],
        "shwfs_addnoise_dev": [vp, vp, C.c_long, vp, vp, vp, C.c_double, C.c_double, C.c_double, C.c_double,
                               C.c_uint64, C.c_uint32, C.c_uint32],
        "shwfs_sync": [vp],
        "shwfs_profile_enable": [vp, i],
        "shwfs_profile_read": [vp, dp, ip],
        "shwfs_copy_counters": [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)],
        "shwfs_autotune": [vp, i, i, i, ip],
        "shwfs_set_variant": [vp, i, i],
        "shwfs_set_trace_order": [vp, i],
        "shwfs_frame_noalloc": [vp, i, i, vp, vp],
        "shwfs_powfs_set_etf_dtrat": [vp, i, i],
        "shwfs_powfs_set_saasum": [vp, i, C.c_double],
        "shwfs_powfs_set_dtrat": [vp, i, i],
        "shwfs_grad_ztilt_dev": [vp, i, vp, vp],
        "shwfs_wfs_set_neasim": [vp, i, dp],
        "shwfs_powfs_set_gs0": [vp, i, i, C.c_long, C.c_long, ip, ip, dp],
        "shwfs_evl_set_aper": [vp, C.c_long, dp, dp, C.c_double, dp],
        "shwfs_evl_add_dir": [vp, C.c_double, C.c_double, C.c_double, ip],
        "shwfs_evl_set_psf": [vp, i, dp, ip, ip, i],
        "shwfs_evl_queue": [vp, i, i],
        "shwfs_evl_sync": [vp, dp, dp],
        "shwfs_evl_psf_get": [vp, i, i, dp, C.POINTER(C.c_long)],
        "shwfs_evl_psf_reset": [vp],
        "shwfs_evl_opd_dev": [vp, i, vp],
        "shwfs_grad_gtilt_dev": [vp, i, vp, vp],
        "shwfs_dm_set": [vp, i, C.POINTER(LayerDesc), C.POINTER(dp)],
        "shwfs_set_worklist": [vp, i, i, i],
        "shwfs_set_branch_priority": [vp, i],
        "shwfs_set_stream_priority": [vp, i],
        "shwfs_autotune_frame": [vp, i, i, i, ip],
        "shwfs_wfs_set_opd_terms": [vp, i, i, dp, C.c_double, C.c_double, dp],
        "shwfs_wfs_set_opdadd": [vp, i, dp],
        "shwfs_powfs_set_seotf": [vp, i, dp],
        "shwfs_wfs_get_mtche": [vp, i, dp, dp, dp],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    lib.shwfs_last_error.argtypes = [vp]
    lib.shwfs_last_error.restype = C.c_char_p
    lib.shwfs_version.argtypes = []
    lib.shwfs_version.restype = C.c_char_p
    lib.shwfs_stream.argtypes = [vp]
    lib.shwfs_stream.restype = vp
    return lib


_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _dptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _devptr(t) -> Optional[int]:
    """Device address of a torch tensor (or an int address)."""
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return int(t.data_ptr())


_live = weakref.WeakSet()


@atexit.register
def _close_all():
    """Close the contexts still open when the interpreter exits, while the
    CUDA runtime is still up (its own exit handlers run after Python's)."""
    for ctx in list(_live):
        try:
            ctx.close()
        except Exception:
            pass


class Context:
    """One device context: static powfs/WFS data, screens and frame buffers."""

    def __init__(self, device: int = 0):
        self._L = lib()
        h = C.c_void_p()
        rc = self._L.shwfs_create(C.byref(h), device)
        if rc != 0:
            raise ShwfsError(f"shwfs_create(device={device}) failed with {rc}")
        self._h = h
        self.npix = {}
        self.nsa = {}
        self.wfs_nsa = {}  # iwfs -> subapertures of its powfs
        self.wfs_powfs = {}  # iwfs -> its powfs
        _live.add(self)

    def _check(self, rc: int, what: str):
        if rc != 0:
            msg = self._L.shwfs_last_error(self._h)
            raise ShwfsError(f"{what}: {msg.decode() if msg else rc} (status {rc})")

    def close(self):
        if getattr(self, "_h", None):
            self._L.shwfs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def stream(self) -> int:
        return int(self._L.shwfs_stream(self._h) or 0)

    # ---- static data ----
    def powfs_add(self, **kw) -> int:
        d = PowfsDesc(**kw)
        out = C.c_int()
        self._check(self._L.shwfs_powfs_add(self._h, C.byref(d), C.byref(out)), "powfs_add")
        self.npix[out.value] = d.pixpsax * d.pixpsay
        self.nsa[out.value] = d.nsa
        return out.value

    def powfs_set_geom(self, ipowfs, origx, origy, amp, saa=None, namp=1):
        ox, oy, am = _f64(origx), _f64(origy), _f64(amp)
        sa = _f64(saa) if saa is not None else None
        self._check(self._L.shwfs_powfs_set_geom(self._h, ipowfs, _dptr(ox), _dptr(oy), _dptr(am), namp, _dptr(sa)),
                    "powfs_set_geom")

    def powfs_set_nominal(self, ipowfs, nominal, nnominal=1):
        a = _f64(nominal)
        self._check(self._L.shwfs_powfs_set_nominal(self._h, ipowfs, _dptr(a), nnominal), "powfs_set_nominal")

    def powfs_set_simap(self, ipowfs, idx, wt, nmap=1):
        ii = np.ascontiguousarray(idx, dtype=np.int32)
        ww = _f64(wt)
        self._check(self._L.shwfs_powfs_set_simap(self._h, ipowfs, ii.ctypes.data_as(C.POINTER(C.c_int)), _dptr(ww),
                                                   nmap), "powfs_set_simap")

    def powfs_set_etf(self, ipowfs, etf, slot=0):
        a = np.ascontiguousarray(etf, dtype=np.complex128).view(np.float64)
        self._check(self._L.shwfs_powfs_set_etf(self._h, ipowfs, _dptr(a), slot), "powfs_set_etf")

    def powfs_set_etf_dtrat(self, ipowfs, dtrat: int):
        """ETF time interpolation: frame isim blends slots 0 and 1 with weight
        (isim mod dtrat) / dtrat on slot 1 (0 turns it off)."""
        self._check(self._L.shwfs_powfs_set_etf_dtrat(self._h, ipowfs, int(dtrat)), "powfs_set_etf_dtrat")

    def powfs_set_gs0(self, ipowfs, nrow, ncol, pp, pi, px, iamp=0):
        """G-tilt operator (MAOS CSC: column pointers pp, row indices pi, values px)."""
        a = np.ascontiguousarray(pp, dtype=np.int32)
        b = np.ascontiguousarray(pi, dtype=np.int32)
        v = _f64(px)
        ipt = C.POINTER(C.c_int)
        self._check(self._L.shwfs_powfs_set_gs0(self._h, ipowfs, iamp, nrow, ncol, a.ctypes.data_as(ipt),
                                                b.ctypes.data_as(ipt), _dptr(v)), "powfs_set_gs0")

    def powfs_set_dtrat(self, ipowfs, dtrat: int):
        """Frames integrated per output frame (noise and gradients on the last)."""
        self._check(self._L.shwfs_powfs_set_dtrat(self._h, ipowfs, int(dtrat)), "powfs_set_dtrat")

    def powfs_set_saasum(self, ipowfs, saasum: float):
        """powfs.saasum for sigmatch 2 CoG (default: the sum of saa)."""
        self._check(self._L.shwfs_powfs_set_saasum(self._h, ipowfs, float(saasum)), "powfs_set_saasum")

    def powfs_set_seotf(self, ipowfs, seotf):
        """Short-exposure OTF per subaperture ((nsa, notf^2) complex, peak in the corner) for the
        device matched-filter regeneration; None removes it."""
        if seotf is None:
            self._check(self._L.shwfs_powfs_set_seotf(self._h, ipowfs, None), "powfs_set_seotf")
            return
        a = np.ascontiguousarray(seotf, dtype=np.complex128).view(np.float64)
        self._check(self._L.shwfs_powfs_set_seotf(self._h, ipowfs, _dptr(a)), "powfs_set_seotf")

    def powfs_set_lltamp(self, ipowfs, lltamp):
        a = _f64(lltamp)
        self._check(self._L.shwfs_powfs_set_lltamp(self._h, ipowfs, _dptr(a)), "powfs_set_lltamp")

    def wfs_add(self, **kw) -> int:
        d = WfsDesc(**kw)
        out = C.c_int()
        self._check(self._L.shwfs_wfs_add(self._h, C.byref(d), C.byref(out)), "wfs_add")
        self.wfs_nsa[out.value] = self.nsa.get(d.ipowfs, 0)
        self.wfs_powfs[out.value] = d.ipowfs
        return out.value

    def wfs_set_mtche(self, iwfs, mtche, i0sum=None, i0sumsum=0.0):
        m = _f64(mtche) if mtche is not None else None
        s = _f64(i0sum) if i0sum is not None else None
        self._check(self._L.shwfs_wfs_set_mtche(self._h, iwfs, _dptr(m), _dptr(s), float(i0sumsum)), "wfs_set_mtche")

    def wfs_set_neasim(self, iwfs, nea):
        """Geometric-gradient noise of WFS iwfs: (3, nsa) or 3*nsa Cholesky
        factor (xx, yy, xy) in radians; None removes it."""
        a = _f64(nea) if nea is not None else None
        self._check(self._L.shwfs_wfs_set_neasim(self._h, iwfs, _dptr(a)), "wfs_set_neasim")

    def wfs_seed(self, iwfs, seed):
        self._check(self._L.shwfs_wfs_seed(self._h, iwfs, int(seed) & 0xFFFFFFFFFFFFFFFF), "wfs_seed")

    def atm_set(self, layers: Sequence[dict], screens: Sequence[np.ndarray]):
        n = len(layers)
        descs = (LayerDesc * max(n, 1))(*[LayerDesc(**l) for l in layers])
        keep = [_f64(s) for s in screens]
        ptrs = (C.POINTER(C.c_double) * max(n, 1))(*[_dptr(s) for s in keep])
        self._check(self._L.shwfs_atm_set(self._h, n, descs, ptrs), "atm_set")

    def dm_set(self, mirrors: Sequence[dict], surfaces: Sequence[np.ndarray]):
        """Deformable-mirror grids subtracted from the OPD of WFS that use them
        (layer dicts: nx, ny, dx, ox, oy, ht, alpha = weight, -1 to subtract;
        surfaces (ny, nx)); later calls with the same sizes copy new surfaces."""
        n = len(mirrors)
        descs = (LayerDesc * max(n, 1))(*[LayerDesc(**{**dict(vx=0.0, vy=0.0), **m}) for m in mirrors])
        keep = [_f64(s) for s in surfaces]
        ptrs = (C.POINTER(C.c_double) * max(n, 1))(*[_dptr(s) for s in keep])
        self._check(self._L.shwfs_dm_set(self._h, n, descs, ptrs), "dm_set")

    def wfs_set_opd_terms(self, iwfs: int, use_dm: bool = False, ptt=(0.0, 0.0, 0.0), focus_tel: float = 0.0,
                          focus_llt: float = 0.0, lltptt=(0.0, 0.0)):
        """Closed-loop terms of WFS iwfs's OPD for the frames queued from now on."""
        p = _f64(ptt)
        lp = _f64(lltptt)
        self._check(self._L.shwfs_wfs_set_opd_terms(self._h, iwfs, int(bool(use_dm)), _dptr(p), float(focus_tel),
                                                    float(focus_llt), _dptr(lp)), "wfs_set_opd_terms")

    def wfs_set_opdadd(self, iwfs: int, opd: Optional[np.ndarray]):
        """NCPA surface (nsa*nopd^2 on the pupil points) added to WFS iwfs's OPD; None removes it."""
        a = _f64(opd).ravel() if opd is not None else None
        self._check(self._L.shwfs_wfs_set_opdadd(self._h, iwfs, _dptr(a)), "wfs_set_opdadd")

    def set_worklist(self, on: bool = True, slices: int = 0, group: int = 0):
        """Imaging of every powfs of a frame as one persistent work-list launch (slices, group: 0
        keeps the current values)."""
        self._check(self._L.shwfs_set_worklist(self._h, int(bool(on)), int(slices), int(group)), "set_worklist")

    def set_branch_priority(self, on: bool = True):
        """Smaller powfs' stream branches at the greatest stream priority (default on)."""
        self._check(self._L.shwfs_set_branch_priority(self._h, int(bool(on))), "set_branch_priority")

    def set_stream_priority(self, priority: int):
        """Priority of the context's streams (lower runs first; clamped to the device's range).
        The stream handle changes: read `stream` again after the call."""
        self._check(self._L.shwfs_set_stream_priority(self._h, int(priority)), "set_stream_priority")

    def set_form(self, form: int):
        self._check(self._L.shwfs_set_form(self._h, form), "set_form")

    def set_dt(self, dt: float):
        self._check(self._L.shwfs_set_dt(self._h, float(dt)), "set_dt")

    # ---- frames ----
    def frame_queue(self, isim: int, iwfs0: int, iwfs1: int):
        self._check(self._L.shwfs_frame_queue(self._h, isim, iwfs0, iwfs1), "frame_queue")

    def frame_sync_range(self, iwfs0: int, iwfs1: int, nsa_of=None, out: Optional[np.ndarray] = None):
        """Gradients of WFS iwfs0..iwfs1-1 after their frame, with one wait.

        With ``out`` (a C-contiguous float64 array of at least the range's
        2 nsa values per WFS, in WFS order) they are written there and ``out``
        is returned: a caller that consumes each frame before the next reuses
        one buffer, as a C caller does.  Otherwise one new array per WFS is
        returned (nsa_of(i), if given, is WFS i's subaperture count)."""
        if out is not None:
            n = 0
            for i in range(iwfs0, iwfs1):
                n += 2 * self.wfs_nsa[i]
            if out.dtype != np.float64 or not out.flags.c_contiguous or out.size < n:
                raise ValueError(f"frame_sync_range: out must be a C-contiguous float64 array of >= {n} values")
            self._check(self._L.shwfs_frame_sync_range(self._h, iwfs0, iwfs1, _dptr(out)), "frame_sync_range")
            return out
        f = nsa_of if nsa_of is not None else self.wfs_nsa.__getitem__
        sizes = [2 * f(i) for i in range(iwfs0, iwfs1)]
        g = np.zeros(sum(sizes))
        self._check(self._L.shwfs_frame_sync_range(self._h, iwfs0, iwfs1, _dptr(g)), "frame_sync_range")
        return np.split(g, np.cumsum(sizes)[:-1])

    def wfs_get_mtche(self, iwfs: int):
        """(mtche (nsa, 2*npix), i0sum (nsa), i0sumsum) held for WFS iwfs."""
        nsa = self.wfs_nsa[iwfs]
        npix = self.npix[self.wfs_powfs[iwfs]]
        m = np.zeros(nsa * 2 * npix)
        s = np.zeros(nsa)
        tot = C.c_double()
        self._check(self._L.shwfs_wfs_get_mtche(self._h, iwfs, _dptr(m), _dptr(s), C.byref(tot)), "wfs_get_mtche")
        return m.reshape(nsa, 2 * npix), s, tot.value

    def wfs_update_mtche(self, iwfs: int, mtchcr: int):
        """Regenerate WFS iwfs's matched filter on the device (shwfs_wfs_update_mtche)."""
        self._check(self._L.shwfs_wfs_update_mtche(self._h, iwfs, mtchcr), "wfs_update_mtche")

    def frame_graph(self, isim: int, iwfs0: int, iwfs1: int):
        """The frame of frame_queue as one CUDA graph (the first call per WFS range runs it plainly)."""
        self._check(self._L.shwfs_frame_graph(self._h, isim, iwfs0, iwfs1), "frame_graph")

    def frame_sync(self, iwfs: int, ipowfs: int, want_ints: bool = False):
        nsa = self.nsa[ipowfs]
        g = np.zeros(2 * nsa)
        ints = np.zeros(nsa * self.npix[ipowfs]) if want_ints else None
        self._check(self._L.shwfs_frame_sync(self._h, iwfs, _dptr(g), _dptr(ints)), "frame_sync")
        return (g, ints) if want_ints else g

    def raytrace_dev(self, iwfs, isim, opd):
        self._check(self._L.shwfs_raytrace_dev(self._h, iwfs, isim, _devptr(opd)), "raytrace_dev")

    def ints_grad_dev(self, iwfs, isim, opd, lltopd=None, ints=None, grad=None, add_noise=False):
        self._check(self._L.shwfs_ints_grad_dev(self._h, iwfs, isim, _devptr(opd), _devptr(lltopd), _devptr(ints),
                                                _devptr(grad), 1 if add_noise else 0), "ints_grad_dev")

    def frame_noalloc(self, iwfs, isim, ints=None, grad=None):
        """One frame of WFS iwfs that allocates no device memory (scratch in a
        static device array); ints/grad are caller-owned device tensors."""
        self._check(self._L.shwfs_frame_noalloc(self._h, iwfs, isim, _devptr(ints), _devptr(grad)), "frame_noalloc")

    def grad_ztilt_dev(self, iwfs, opd, grad):
        """Geometric z-tilt gradients (2*nsa, device) of a device OPD (nsa*nopd^2)."""
        self._check(self._L.shwfs_grad_ztilt_dev(self._h, iwfs, _devptr(opd), _devptr(grad)), "grad_ztilt_dev")

    def grad_gtilt_dev(self, iwfs, opd, grad):
        """G-tilt gradients GS0 opd (2*nsa, device) of a device OPD."""
        self._check(self._L.shwfs_grad_gtilt_dev(self._h, iwfs, _devptr(opd), _devptr(grad)), "grad_gtilt_dev")

    def grad_dev(self, iwfs, ints, grad):
        self._check(self._L.shwfs_grad_dev(self._h, iwfs, _devptr(ints), _devptr(grad)), "grad_dev")

    def addnoise_dev(self, ints, seed: int, stream: int = 0, frame: int = 0, bkgrnd: float = 0.0,
                     bkgrndc: float = 0.0, rne: float = 0.0, excess: float = 1.0, bkgrnd2=None, bkgrnd2c=None, qe=None):
        """Photon and read noise in place on a CUDA float32 tensor (addnoise, lib/libmisc.c:31)."""
        self._check(self._L.shwfs_addnoise_dev(self._h, _devptr(ints), ints.numel(), _devptr(bkgrnd2),
                                               _devptr(bkgrnd2c), _devptr(qe), bkgrnd, bkgrndc, rne, excess,
                                               seed, stream, frame), "addnoise_dev")

    # ---- science path (include/shwfs_evl.h) ----
    def evl_set_aper(self, locx, locy, dx, amp):
        x, y, a = _f64(locx), _f64(locy), _f64(amp)
        self._check(self._L.shwfs_evl_set_aper(self._h, len(x), _dptr(x), _dptr(y), float(dx), _dptr(a)),
                    "evl_set_aper")
        self._evl_n = 0

    def evl_add_dir(self, thetax, thetay, hs=math.inf) -> int:
        out = C.c_int()
        self._check(self._L.shwfs_evl_add_dir(self._h, float(thetax), float(thetay), float(hs), C.byref(out)),
                    "evl_add_dir")
        self._evl_n = out.value + 1
        return out.value

    def evl_set_psf(self, wvl, nembed, psfsize=None, pttr=False):
        w = _f64(wvl)
        n = np.ascontiguousarray(nembed, dtype=np.int32)
        p = np.ascontiguousarray(psfsize if psfsize is not None else [0] * len(w), dtype=np.int32)
        ipt = C.POINTER(C.c_int)
        self._check(self._L.shwfs_evl_set_psf(self._h, len(w), _dptr(w), n.ctypes.data_as(ipt), p.ctypes.data_as(ipt),
                                              1 if pttr else 0), "evl_set_psf")
        self._evl_psfsize = [int(q if q > 0 else m) for q, m in zip(p, n)]

    def evl_queue(self, isim: int, do_psf: bool = False):
        self._check(self._L.shwfs_evl_queue(self._h, int(isim), 1 if do_psf else 0), "evl_queue")

    def evl_sync(self):
        """(wfe, coeff), each (nevl, 3): {PR, TT, PTTR} and {piston, tip, tilt}."""
        n = getattr(self, "_evl_n", 0)
        wfe, coeff = np.zeros(3 * n), np.zeros(3 * n)
        self._check(self._L.shwfs_evl_sync(self._h, _dptr(wfe), _dptr(coeff)), "evl_sync")
        return wfe.reshape(n, 3), coeff.reshape(n, 3)

    def evl_psf(self, ievl: int, iwvl: int):
        """(psf (psfsize, psfsize) with psf[ix, iy], number of frames summed)."""
        n = self._evl_psfsize[iwvl]
        out = np.zeros(n * n)
        nf = C.c_long()
        self._check(self._L.shwfs_evl_psf_get(self._h, ievl, iwvl, _dptr(out), C.byref(nf)), "evl_psf_get")
        return out.reshape(n, n, order="F"), nf.value

    def evl_psf_reset(self):
        self._check(self._L.shwfs_evl_psf_reset(self._h), "evl_psf_reset")

    def evl_opd_dev(self, ievl: int, opd):
        self._check(self._L.shwfs_evl_opd_dev(self._h, ievl, _devptr(opd)), "evl_opd_dev")

    def sync(self):
        self._check(self._L.shwfs_sync(self._h), "sync")

    def copy_counters(self):
        """(host->device bytes, device->host bytes) copied on the frame path since the last call."""
        a, b = C.c_uint64(), C.c_uint64()
        self._check(self._L.shwfs_copy_counters(self._h, C.byref(a), C.byref(b)), "copy_counters")
        return a.value, b.value

    def autotune(self, iwfs0: int, iwfs1: int, nrep: int = 5) -> int:
        """Pick the fastest imaging-kernel variant on the real frames; returns its index."""
        out = C.c_int()
        self._check(self._L.shwfs_autotune(self._h, iwfs0, iwfs1, nrep, C.byref(out)), "autotune")
        return out.value

    def autotune_frame(self, iwfs0: int, iwfs1: int, nrep: int = 5) -> int:
        """Per-powfs launches or the work list (and its settings), whichever runs the frame
        fastest; returns the choice (0: per-powfs launches)."""
        out = C.c_int()
        self._check(self._L.shwfs_autotune_frame(self._h, iwfs0, iwfs1, nrep, C.byref(out)), "autotune_frame")
        return out.value

    def set_variant(self, ipowfs: int, variant: int):
        self._check(self._L.shwfs_set_variant(self._h, ipowfs, variant), "set_variant")

    def set_trace_order(self, order: int):
        """Pupil order of ray-trace launches (SHWFS_TRACE_AUTO, _LISTED, _INTERLEAVED)."""
        self._check(self._L.shwfs_set_trace_order(self._h, order), "set_trace_order")

    STAGES = ("raytrace", "uplink", "ints", "post")

    def profile_enable(self, on: bool = True):
        self._check(self._L.shwfs_profile_enable(self._h, 1 if on else 0), "profile_enable")

    def profile_read(self):
        """{stage: (device ms summed, launches)} since the previous read."""
        ms = (C.c_double * len(self.STAGES))()
        n = (C.c_int * len(self.STAGES))()
        self._check(self._L.shwfs_profile_read(self._h, ms, n), "profile_read")
        return {k: (ms[i], n[i]) for i, k in enumerate(self.STAGES)}


def version() -> str:
    return lib().shwfs_version().decode()
