"""Geometric (z-tilt) gradients and ETF time interpolation on the GPU, against
the reference's own CPU code (oracle/_ref):

- z-tilt of a device OPD against pts_mcc_ptt / dcellinvspd_each / pts_ztilt
  (maos/powfs.c:633-645, math/loc.c:839-885) on the same OPD;
- G-tilt of a device OPD against the reference's mkg operator GS0
  (lib/mkg.c:471, maos/powfs.c:619-626) applied by its dspmm;
- full frames of geometric sensors (ray trace + z-tilt or G-tilt) against
  the reference's prop + pts_ztilt / GS0 on the same screens;
- the noise of geometric gradients (add_geom_noise_do,
  cuda/sim/wfsgrad.cu:39-51): sample covariance against L L^T;
- LGS frames with two ETFs interpolated in time (maos/wfsints.c:215-223)
  against the reference's wfsints with etfsim2 and coldtrat.

Tolerances: gradients within 1e-5 relative (max |dg| / max |g|) from a
shared FP32 OPD, 1e-4 from independently traced OPDs; intensities within
1e-5 of the subaperture total."""
import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def _geom_ctx(ref_lib, cfg, thetas, noisy=0, nx=512, seed=3, gradtype=None):
    """A context with one geometric powfs of the reference's geometry (and,
    for G-tilt, its GS0) and a WFS per direction, under the turbulence of the
    workload builder."""
    from maos_b200 import shwfs
    from maos_b200.workload import build
    wl = build(cfg, device=0, seed=seed, noisy=False, nx=nx)  # for its screens and layers
    r = ref_lib.RefPowfs(cfg)
    ctx = shwfs.Context(0)
    ctx.set_dt(cfg["dt"])
    gt = shwfs.SHWFS_GRAD_ZTILT if gradtype is None else gradtype
    ip = ctx.powfs_add(nsa=r.nsa, nopd=r.nopd, embfac=1, notf=0, pixpsax=0, pixpsay=0, dsa=cfg["dsa"],
                       dx=r.ptsdx(), hs=cfg["hs"], areascale=1.0, wvl=cfg["wvl"], gradtype=gt)
    ox, oy = r.ptsorig()
    ctx.powfs_set_geom(ip, ox, oy, r.amp())
    if gt == shwfs.SHWFS_GRAD_GTILT:
        ctx.powfs_set_gs0(ip, *r.gs0())
    ws = []
    for k, (tx, ty) in enumerate(thetas):
        i = ctx.wfs_add(ipowfs=ip, thetax=tx, thetay=ty, hs=cfg["hs"], hc=0.0, misregx=0.0, misregy=0.0,
                        sigsim=1.0, wvlwt=1.0, noisy=noisy)
        ctx.wfs_seed(i, 77 + k)
        ws.append(i)
    ctx.atm_set(wl.layers, wl.screens)
    return ctx, ip, ws, wl, r


def _rel(g, g_ref):
    return np.abs(g - g_ref).max() / np.abs(g_ref).max()


def test_ztilt_dev_matches_reference(ref_lib):
    import torch
    from maos_b200.configs import NGS8
    from maos_b200.workload import build
    wl = build(NGS8, device=0, seed=5, noisy=False, nx=512)
    r = ref_lib.RefPowfs(NGS8)
    iw = wl.wfs[0]
    opd = torch.zeros(r.nsa * r.nopd ** 2, dtype=torch.float32, device="cuda")
    grad = torch.zeros(2 * r.nsa, dtype=torch.float32, device="cuda")
    wl.ctx.raytrace_dev(iw, 11, opd)
    wl.ctx.grad_ztilt_dev(iw, opd, grad)
    wl.ctx.sync()
    g_ref = r.ztilt(opd.double().cpu().numpy())
    assert _rel(grad.double().cpu().numpy(), g_ref) <= 1e-5
    wl.close()


def test_gtilt_dev_matches_reference(ref_lib):
    import torch
    from maos_b200 import shwfs
    from maos_b200.configs import NGS8
    ctx, ip, ws, wl, r = _geom_ctx(ref_lib, NGS8, [(0.0, 0.0)], gradtype=shwfs.SHWFS_GRAD_GTILT)
    opd = torch.zeros(r.nsa * r.nopd ** 2, dtype=torch.float32, device="cuda")
    grad = torch.zeros(2 * r.nsa, dtype=torch.float32, device="cuda")
    ctx.raytrace_dev(ws[0], 17, opd)
    ctx.grad_gtilt_dev(ws[0], opd, grad)
    ctx.sync()
    g_ref = r.gtilt(opd.double().cpu().numpy())
    assert _rel(grad.double().cpu().numpy(), g_ref) <= 1e-5
    ctx.close()
    wl.close()


@pytest.mark.parametrize("isim", [0, 41])
@pytest.mark.parametrize("kind", ["ztilt", "gtilt"])
def test_geometric_frame_matches_reference(ref_lib, isim, kind):
    from maos_b200 import shwfs
    from maos_b200.configs import NGS8
    thetas = [(NGS8["thetax"][0], NGS8["thetay"][0]), (3e-5, -2e-5)]
    gt = shwfs.SHWFS_GRAD_ZTILT if kind == "ztilt" else shwfs.SHWFS_GRAD_GTILT
    ctx, ip, ws, wl, r = _geom_ctx(ref_lib, NGS8, thetas, gradtype=gt)
    ctx.frame_queue(isim, ws[0], ws[-1] + 1)
    out = ctx.frame_sync_range(ws[0], ws[-1] + 1, lambda i: r.nsa)
    dt = NGS8["dt"]
    for k, (tx, ty) in enumerate(thetas):
        opd_ref = np.zeros(r.nsa * r.nopd ** 2)
        for L, scr in zip(wl.layers, wl.screens):
            r.prop_layer(scr, L["dx"], L["ox"], L["oy"], L["ht"], tx, ty, NGS8["hs"], -L["vx"] * dt * isim,
                         -L["vy"] * dt * isim, opd=opd_ref)
        g_ref = r.ztilt(opd_ref) if kind == "ztilt" else r.gtilt(opd_ref)
        assert _rel(out[k], g_ref) <= 1e-4, (k, _rel(out[k], g_ref))
    with pytest.raises(Exception):
        ctx.frame_sync(ws[0], ip, want_ints=True)  # no pixels on a geometric sensor
    ctx.close()
    wl.close()


def test_geometric_noise_covariance():
    """Noisy minus noise-free gradients of two WFS in the same direction:
    zero mean and covariance L L^T, L = [[nea_xx, 0], [nea_xy, nea_yy]]."""
    from oracle import ref as ref_lib
    if not ref_lib.available():
        pytest.skip("oracle/_ref is not built")
    from maos_b200.configs import NGS8
    th = (NGS8["thetax"][0], NGS8["thetay"][0])
    ctx, ip, ws, wl, r = _geom_ctx(ref_lib, NGS8, [th, th], noisy=1)
    nsa = r.nsa
    lxx, lyy, lxy = 2e-7, 3e-7, -1e-7
    ctx.wfs_set_neasim(ws[0], np.concatenate([np.full(nsa, lxx), np.full(nsa, lyy), np.full(nsa, lxy)]))
    d = []
    for isim in range(300):
        ctx.frame_queue(isim, ws[0], ws[-1] + 1)
        g1, g0 = ctx.frame_sync_range(ws[0], ws[-1] + 1, lambda i: nsa)
        d.append(np.stack([g1[:nsa] - g0[:nsa], g1[nsa:] - g0[nsa:]], axis=1))
    n = np.concatenate(d)  # (frames * nsa, 2)
    cov = np.cov(n.T)
    want = np.array([[lxx * lxx, lxx * lxy], [lxx * lxy, lxy * lxy + lyy * lyy]])
    m = len(n)
    assert np.abs(n.mean(axis=0)).max() <= 5 * np.sqrt(want.diagonal().max() / m)
    assert np.abs(cov - want).max() <= 6 * want.max() * np.sqrt(2.0 / m), (cov, want)
    # noise is keyed by (seed, subaperture, WFS, frame): the same frame repeats exactly
    ctx.frame_queue(5, ws[0], ws[-1] + 1)
    a = ctx.frame_sync_range(ws[0], ws[-1] + 1, lambda i: nsa)[0]
    ctx.frame_queue(5, ws[0], ws[-1] + 1)
    b = ctx.frame_sync_range(ws[0], ws[-1] + 1, lambda i: nsa)[0]
    assert np.array_equal(a, b)
    ctx.close()
    wl.close()


@pytest.mark.parametrize("isim", [5, 6, 8])
def test_etf_time_interpolation_matches_reference(ref_lib, isim):
    from maos_b200.configs import LGS30
    from tests.helpers import ints_tolerance_ok, grad_rel_err
    from maos_b200.workload import build
    dtrat = 4
    wl = build(LGS30, device=0, seed=3, noisy=False, nx=512)
    r = ref_lib.RefPowfs(LGS30)
    r.setup_etf2(1500.0, dtrat)
    for i in wl.wfs:
        wl.ctx.wfs_set_mtche(i, r.mtche(), r.i0sum(), r.i0sumsum())
    wl.ctx.powfs_set_etf(wl.ipowfs, r.etf(), slot=0)
    wl.ctx.powfs_set_etf(wl.ipowfs, r.etf2(), slot=1)
    wl.ctx.powfs_set_etf_dtrat(wl.ipowfs, dtrat)
    ref_lib.atm_set(wl.screens, wl.layers)
    wl.frame(isim)
    out = wl.frame_sync(want_ints=True)
    for k in (0, 4):
        ints_ref, g_ref, _ = ref_lib.frame_full_mt(r, k, isim, LGS30["dt"], noisy=False)
        g, ints = out[k]
        ok, worst = ints_tolerance_ok(ints, ints_ref, r.nsa, r.npix, 1e-5)
        assert ok, f"wfs {k}: intensity error {worst:.3e} of subaperture total"
        assert grad_rel_err(g, g_ref) <= 1e-4, (k, grad_rel_err(g, g_ref))
    if isim % dtrat:
        # the interpolated frame differs from slot 0 alone
        wl.ctx.powfs_set_etf_dtrat(wl.ipowfs, 0)
        wl.frame(isim)
        g0 = wl.frame_sync()[0]
        assert grad_rel_err(g0, out[0][0]) > 1e-3
    wl.close()


@pytest.mark.parametrize("size,form", [(64, "fft"), (128, "fft"), (32, "tc")])
def test_etf_time_interpolation_in_every_imaging_path(ref_lib, size, form):
    """The two-slot ETF blend (maos/wfsints.c:212-221, 282) in the 64-point fused kernel, the
    FFT-pass chain (FFT 128) and the tensor-core form, each against the reference's frame with
    its second sodium profile, at a frame that weights both slots 1/2."""
    from maos_b200 import shwfs
    from maos_b200.configs import LGS8_N32, LGS8_N64
    from maos_b200.workload import build
    from tests.helpers import ints_tolerance_ok, grad_rel_err
    cfg = {32: LGS8_N32, 64: LGS8_N64,
           128: dict(LGS8_N64, name="lgs8_2x8x8_n128", embfac=4, notf=128, pixpsa=8)}[size]
    f = shwfs.SHWFS_FORM_TC if form == "tc" else shwfs.SHWFS_FORM_FFT
    dtrat, isim = 4, 6
    wl = build(cfg, device=0, seed=3, noisy=False, nx=512, form=f)
    r = ref_lib.RefPowfs(cfg)
    r.setup_etf2(1500.0, dtrat)
    for i in wl.wfs:
        wl.ctx.wfs_set_mtche(i, r.mtche(), r.i0sum(), r.i0sumsum())
    wl.ctx.powfs_set_etf(wl.ipowfs, r.etf(), slot=0)
    wl.ctx.powfs_set_etf(wl.ipowfs, r.etf2(), slot=1)
    wl.ctx.powfs_set_etf_dtrat(wl.ipowfs, dtrat)
    ref_lib.atm_set(wl.screens, wl.layers)
    wl.frame(isim)
    out = wl.frame_sync(want_ints=True)
    tol = 1e-4 if form == "tc" else 1e-5
    for k in range(len(wl.wfs)):
        ints_ref, g_ref, _ = ref_lib.frame_full_mt(r, k, isim, cfg["dt"], noisy=False)
        g, ints = out[k]
        ok, worst = ints_tolerance_ok(ints, ints_ref, r.nsa, r.npix, tol)
        assert ok, f"wfs {k}: intensity error {worst:.3e} of subaperture total"
        assert grad_rel_err(g, g_ref) <= 1e-4, (k, grad_rel_err(g, g_ref))
    wl.close()
