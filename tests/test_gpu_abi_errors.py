"""Error behaviour of the C ABI on a GPU: invalid arguments and calls out of
order return the documented status (SHWFS_EINVAL -1, SHWFS_ESTATE -3) with a
message from shwfs_last_error, and leave the context usable."""
import ctypes as C
import math

import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

EINVAL, ESTATE = -1, -3


def _desc(**kw):
    d = dict(nsa=4, nopd=16, embfac=2, notf=32, pixpsax=6, pixpsay=6, pixthetax=1e-6, pixthetay=1e-6, wvl=5e-7,
             dsa=0.5, dx=1 / 32, areascale=1.0, hs=math.inf, gradtype=2, sigmatch=1, saat=0.3, sigtot_cog=1000.0)
    d.update(kw)
    return d


def _rc(ctx, fn, *args):
    return getattr(ctx._L, fn)(ctx._h, *args)


def test_invalid_powfs_descriptors():
    from maos_b200 import shwfs
    ctx = shwfs.Context(0)
    bad = [dict(nopd=12), dict(notf=48, embfac=3), dict(pixpsax=12, pixpsay=12), dict(gradtype=7),
           dict(sigmatch=3), dict(nsa=0), dict(has_llt=1, llt_nx=8)]
    for b in bad:
        d = shwfs.PowfsDesc(**_desc(**b))
        out = C.c_int()
        assert ctx._L.shwfs_powfs_add(ctx._h, C.byref(d), C.byref(out)) == EINVAL, b
        assert ctx._L.shwfs_last_error(ctx._h)  # a message
    # the context still works
    ip = ctx.powfs_add(**_desc())
    assert ip == 0
    ctx.close()


def test_calls_out_of_order_and_bad_indices():
    from maos_b200 import shwfs
    ctx = shwfs.Context(0)
    ip = ctx.powfs_add(**_desc())
    iw = ctx.wfs_add(ipowfs=ip, thetax=0.0, thetay=0.0, hs=math.inf, hc=0.0, misregx=0.0, misregy=0.0, sigsim=1000.0,
                     wvlwt=1.0, noisy=0)
    # no geometry, pixel map or DTF yet: the frame is refused, not run
    assert _rc(ctx, "shwfs_frame_queue", 0, iw, iw + 1) == ESTATE
    assert b"not set" in ctx._L.shwfs_last_error(ctx._h)
    assert _rc(ctx, "shwfs_frame_queue", 0, iw, iw + 5) == EINVAL          # WFS range past the end
    assert _rc(ctx, "shwfs_wfs_seed", 99, C.c_uint64(1)) == EINVAL        # unknown WFS
    assert _rc(ctx, "shwfs_powfs_set_etf", 5, None, 0) == EINVAL          # unknown powfs
    assert _rc(ctx, "shwfs_powfs_set_dtrat", ip, 0) == EINVAL
    assert _rc(ctx, "shwfs_evl_queue", 0, 0) == ESTATE                    # no science aperture
    with pytest.raises(shwfs.ShwfsError):
        ctx.evl_sync()
    ctx.sync()
    ctx.close()


def test_gs0_and_geometric_errors():
    from maos_b200 import shwfs
    ctx = shwfs.Context(0)
    ip = ctx.powfs_add(nsa=2, nopd=4, embfac=1, notf=0, pixpsax=0, pixpsay=0, dsa=0.5, dx=0.125, hs=math.inf,
                       areascale=1.0, wvl=5e-7, gradtype=shwfs.SHWFS_GRAD_GTILT)
    ctx.powfs_set_geom(ip, [0.0, 0.5], [0.0, 0.0], np.ones(32))
    pp = np.array([0] * 33, dtype=np.int32)
    # GS0 of the wrong shape, then a row index out of range
    with pytest.raises(shwfs.ShwfsError):
        ctx.powfs_set_gs0(ip, 3, 32, pp, np.zeros(0, np.int32), np.zeros(0))
    pp2 = pp.copy()
    pp2[1:] = 1
    with pytest.raises(shwfs.ShwfsError):
        ctx.powfs_set_gs0(ip, 4, 32, pp2, np.array([9], np.int32), np.array([1.0]))
    iw = ctx.wfs_add(ipowfs=ip, thetax=0.0, thetay=0.0, hs=math.inf, hc=0.0, misregx=0.0, misregy=0.0, sigsim=1.0,
                     wvlwt=1.0, noisy=0)
    # no GS0 yet: the frame is refused
    assert _rc(ctx, "shwfs_frame_queue", 0, iw, iw + 1) == ESTATE
    with pytest.raises(shwfs.ShwfsError):
        ctx.frame_sync(iw, ip, want_ints=True)  # a geometric sensor has no pixels
    ctx.close()
