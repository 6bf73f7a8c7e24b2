"""Ray-trace launches give the same frames in every pupil order: WFS pupils
interleaved (and, for the FFT-64 LGS sensor, its LLT pupils in a second
launch) against the listed order, bit for bit, and the science path's
interleaved directions against the listed order (OPD and PSF bit for bit,
the FP64 wavefront-error sums to their accumulation order)."""
import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def _frames(cfg, order, isims):
    from maos_b200.workload import build
    wl = build(cfg, device=0, seed=5, noisy=True, nx=256)
    wl.ctx.set_trace_order(order)
    out = []
    for isim in isims:
        wl.frame(isim)
        out.append(wl.frame_sync(want_ints=True))
    wl.close()
    return out


@pytest.mark.parametrize("case", ["lgs8_n32", "lgs8_n64", "ngs8"])
def test_interleaved_trace_equals_listed(case):
    from maos_b200 import shwfs
    from maos_b200.configs import LGS8_N32, LGS8_N64, NGS8
    cfg = {"lgs8_n32": LGS8_N32, "lgs8_n64": LGS8_N64, "ngs8": NGS8}[case]
    isims = [0, 3]
    a = _frames(cfg, shwfs.SHWFS_TRACE_LISTED, isims)
    b = _frames(cfg, shwfs.SHWFS_TRACE_INTERLEAVED, isims)
    for fa, fb in zip(a, b):
        for (ga, ia), (gb, ib) in zip(fa, fb):
            assert np.array_equal(ga, gb) and np.array_equal(ia, ib)


def test_science_directions_in_either_order():
    import torch
    from maos_b200 import shwfs
    from maos_b200.configs import LGS8_N32
    from maos_b200.setup import aperture, screens
    from maos_b200.workload import wind
    cfg = LGS8_N32
    at = cfg["atm"]
    nx = 256
    scr = screens(nx, nx, at["dx"], at["r0"], at["L0"], at["wt"], 2)
    vx, vy = wind(cfg, 2)
    o = -nx / 2 * at["dx"]
    layers = [dict(nx=nx, ny=nx, dx=at["dx"], ox=o, oy=o, ht=float(h), vx=float(vx[i]), vy=float(vy[i]), alpha=1.0)
              for i, h in enumerate(at["ht"])]
    x, y, a = aperture(8.0, 1.2, 1.0 / 32)
    res = []
    for order in (shwfs.SHWFS_TRACE_LISTED, shwfs.SHWFS_TRACE_INTERLEAVED):
        ctx = shwfs.Context(0)
        ctx.set_trace_order(order)
        ctx.set_dt(cfg["dt"])
        ctx.atm_set(layers, scr)
        ctx.evl_set_aper(x, y, 1.0 / 32, a)
        for tx, ty in ((0.0, 0.0), (5e-5, 0.0), (0.0, -5e-5)):
            ctx.evl_add_dir(tx, ty, float("inf"))
        # without tip/tilt removal the PSF does not depend on the FP64 sums, whose
        # atomic accumulation order varies from run to run
        ctx.evl_set_psf([1.65e-6], [512], [128], pttr=0)
        ctx.evl_queue(3, do_psf=True)
        wfe, _ = ctx.evl_sync()
        opd = torch.zeros(len(x), dtype=torch.float32, device="cuda")
        ctx.evl_opd_dev(2, opd)
        ctx.sync()
        res.append((np.array(wfe), opd.cpu().numpy(), ctx.evl_psf(1, 0)[0]))
        ctx.close()
    (w0, o0, p0), (w1, o1, p1) = res
    assert np.array_equal(o0, o1) and np.array_equal(p0, p1)
    assert np.allclose(w0, w1, rtol=1e-12, atol=0)


def test_trace_order_rejects_unknown_order():
    from maos_b200 import shwfs
    ctx = shwfs.Context(0)
    with pytest.raises(shwfs.ShwfsError):
        ctx.set_trace_order(3)
    ctx.close()
