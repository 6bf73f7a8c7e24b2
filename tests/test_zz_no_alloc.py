"""The allocation-free frame (shwfs_frame_noalloc) against the ordinary frame.

Some callers cannot allocate device memory once they run: a real-time loop
that forbids allocation after start-up (cudaMalloc can block for a long time
and can fail when memory runs short), or a host application whose device
memory belongs to its own pool.  For them the C ABI has one entry point whose
scratch lives in a static device array.
This test calls it through the C ABI twice in a row and checks each result
against the ordinary entry point (shwfs_frame_queue + shwfs_frame_sync) with
the tolerances of the other parity tests: intensities within 1e-5 of the
subaperture total, gradients within 1e-4 relative.  It lives in a file of its
own that pytest collects last."""
import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def _check(ctx, wl, iwfs, isim):
    import torch
    from tests.helpers import ints_tolerance_ok, grad_rel_err
    wl.frame(isim)
    ref = wl.frame_sync(want_ints=True)
    g_ref, ints_ref = ref[wl.wfs.index(iwfs)]
    dev = torch.device("cuda", 0)
    ints = torch.full((wl.nsa * wl.npix,), float("nan"), dtype=torch.float32, device=dev)
    grad = torch.full((2 * wl.nsa,), float("nan"), dtype=torch.float32, device=dev)
    ctx.frame_noalloc(iwfs, isim, ints, grad)
    ctx.sync()
    ints_h = ints.double().cpu().numpy()
    g_h = grad.double().cpu().numpy()
    ok, worst = ints_tolerance_ok(ints_h, ints_ref, wl.nsa, wl.npix, 1e-5)
    assert ok, f"intensity error {worst:.3e} of subaperture total"
    assert grad_rel_err(g_h, g_ref) <= 1e-4


@pytest.mark.parametrize("cfgname", ["lgs30_6x60x60_mf", "ngs8_16x16_cog"])
def test_noalloc_frame_matches_ordinary_frame_twice(cfgname):
    from maos_b200.configs import CONFIGS
    from maos_b200.workload import build
    cfg = CONFIGS[cfgname]
    wl = build(cfg, device=0, seed=5, noisy=False, nx=512)
    ctx = wl.ctx
    # two calls in a row, different WFS and frames, sharing the static scratch
    _check(ctx, wl, wl.wfs[-1], 11)
    _check(ctx, wl, wl.wfs[0], 12)
    wl.close()


def test_noalloc_rejects_oversized_wfs():
    import torch
    from maos_b200 import shwfs
    ctx = shwfs.Context(0)
    ip = ctx.powfs_add(nsa=5000, nopd=16, embfac=2, notf=32, pixpsax=6,
                       pixpsay=6, pixthetax=4.8e-6, pixthetay=4.8e-6, wvl=0.589e-6, dsa=0.5, dx=1 / 32,
                       areascale=1.0, hs=float("inf"), gradtype=shwfs.SHWFS_GRAD_COG, sigmatch=1, saat=0.3,
                       sigtot_cog=500.0)
    iw = ctx.wfs_add(ipowfs=ip, hs=float("inf"), sigsim=500.0, wvlwt=1.0)
    grad = torch.zeros(2 * 5000, dtype=torch.float32, device="cuda")
    with pytest.raises(shwfs.ShwfsError, match="exceed the allocation-free maximum"):
        ctx.frame_noalloc(iw, 0, None, grad)  # rejected on the host before any launch
    ctx.close()


def _small_powfs(ctx, **over):
    from maos_b200 import shwfs
    kw = dict(nsa=4, nopd=16, embfac=2, notf=32, pixpsax=6, pixpsay=6, pixthetax=4.8e-6, pixthetay=4.8e-6,
              wvl=0.589e-6, dsa=0.5, dx=1 / 32, areascale=1.0, hs=float("inf"), gradtype=shwfs.SHWFS_GRAD_COG,
              sigmatch=1, saat=0.3, sigtot_cog=500.0)
    kw.update(over)
    ip = ctx.powfs_add(**kw)
    return ip, ctx.wfs_add(ipowfs=ip, hs=float("inf"), sigsim=500.0, wvlwt=1.0)


@pytest.mark.parametrize("form", ["fft64_opd16", "fft64_opd8", "dtrat2"])
def test_noalloc_rejects_other_forms(form):
    """Only the 32-point form (16x16 OPD points, 32x32 FFT) runs without
    allocation; a 64-point powfs whose pupil still fits 16x16 points and a
    powfs integrating over frames are refused on the host, before any launch."""
    import torch
    from maos_b200 import shwfs
    ctx = shwfs.Context(0)
    if form == "fft64_opd16":
        ip, iw = _small_powfs(ctx, nopd=16, embfac=4, notf=64)
        msg = "only 16x16 OPD points with a 32x32 FFT"
    elif form == "fft64_opd8":
        ip, iw = _small_powfs(ctx, nopd=8, embfac=8, notf=64)
        msg = "only 16x16 OPD points with a 32x32 FFT"
    else:
        ip, iw = _small_powfs(ctx)
        ctx.powfs_set_dtrat(ip, 2)
        msg = "dtrat > 1"
    grad = torch.zeros(8, dtype=torch.float32, device="cuda")
    with pytest.raises(shwfs.ShwfsError, match=msg):
        ctx.frame_noalloc(iw, 0, None, grad)
    ctx.close()
