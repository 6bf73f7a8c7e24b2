"""Polychromatic sensors: a powfs imaged at several wavelengths (the reference's
loop over powfs.wvl, maos/wfsints.c:145-288) through wavelength bands
(shwfs_powfs_add_band), against the reference's CPU frame of the same
two-wavelength powfs on the same screens.

Tolerances as the other frame tests: noise-free intensities within 1e-5 of the
subaperture total (1e-4 for the tensor-core form); gradients within 1e-4
relative."""
import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


@pytest.mark.parametrize("cfg_name,form,isim", [("NGS8_2WVL", 0, 3), ("LGS8_N32_2WVL", 0, 5), ("NGS8_2WVL", 1, 2),
                                               ("LGS8_N64_2WVL", 0, 4)])
def test_two_wavelength_frame_matches_reference(ref_lib, cfg_name, form, isim):
    from maos_b200 import configs
    from maos_b200.workload import build
    from tests.helpers import ints_tolerance_ok, grad_rel_err
    cfg = getattr(configs, cfg_name)
    wl = build(cfg, device=0, seed=4, noisy=False, nx=512, form=form)
    r = ref_lib.RefPowfs(cfg)
    if cfg["phytype"] == 1:  # the reference's filter, built from its polychromatic i0
        for i in wl.wfs:
            wl.ctx.wfs_set_mtche(i, r.mtche(), r.i0sum(), r.i0sumsum())
    ref_lib.atm_set(wl.screens, wl.layers)
    wl.frame(isim)
    out = wl.frame_sync(want_ints=True)
    tol = 1e-4 if form == 1 else 1e-5
    for k in range(len(wl.wfs)):
        ints_ref, g_ref, _ = ref_lib.frame_full_mt(r, k, isim, cfg["dt"], noisy=False)
        g, ints = out[k]
        ok, worst = ints_tolerance_ok(ints, ints_ref, r.nsa, r.npix, tol)
        assert ok, f"wfs {k}: intensity error {worst:.3e} of subaperture total"
        assert grad_rel_err(g, g_ref) <= 1e-4, (k, grad_rel_err(g, g_ref))
    wl.close()


def test_bands_change_the_image_and_keep_noise_once():
    """The second band adds light: the two-band intensities exceed the first band's alone by the
    second band's weighted image; a noisy frame adds noise once (finite, integer photon counts
    plus read noise), and frames repeat bit for bit."""
    from maos_b200.configs import NGS8_2WVL
    from maos_b200.workload import build
    one = build(dict(NGS8_2WVL, wvls=[0.7e-6], wvlwts=[0.6]), device=0, seed=4, noisy=False, nx=256)
    two = build(NGS8_2WVL, device=0, seed=4, noisy=False, nx=256)
    one.frame(1)
    two.frame(1)
    i1 = one.frame_sync(want_ints=True)[0][1]
    i2 = two.frame_sync(want_ints=True)[0][1]
    assert (i2 >= i1 - 1e-3 * i1.max()).all() and i2.sum() > i1.sum() * 1.2
    one.close()
    two.close()
    a = build(NGS8_2WVL, device=0, seed=4, noisy=True, nx=256)
    a.frame(7)
    g1 = a.frame_sync()
    a.frame(7)
    g2 = a.frame_sync()
    assert all(np.array_equal(x, y) and np.isfinite(x).all() for x, y in zip(g1, g2))
    a.close()


def test_band_arguments_are_checked():
    """A band must keep its powfs' sizes, pixels and options; WFS, dtrat and the device
    matched-filter regeneration belong to the main powfs."""
    from maos_b200 import shwfs
    from maos_b200.configs import NGS8_2WVL
    from maos_b200.setup import Setup
    from maos_b200.workload import build
    wl = build(NGS8_2WVL, device=0, seed=4, noisy=False, nx=256)
    ctx = wl.ctx
    ib = max(ctx.npix)  # the band added by build
    with pytest.raises(shwfs.ShwfsError):
        ctx.wfs_add(ipowfs=ib, thetax=0.0, thetay=0.0, hs=np.inf, hc=0.0, misregx=0.0, misregy=0.0, sigsim=1.0,
                    wvlwt=1.0, noisy=0)
    with pytest.raises(shwfs.ShwfsError):
        ctx.powfs_set_dtrat(ib, 2)
    with pytest.raises(shwfs.ShwfsError):  # other pixels: not a band of this powfs
        s = Setup(dict(NGS8_2WVL, pixpsa=6))
        try:
            s.load_band(ctx, wl.ipowfs, 0.5)
        finally:
            s.close()
    wl.close()


def test_lgs_bands_refuse_the_device_input_path():
    """An LGS powfs with bands forms each band's uplink OTF in the frame path; the single-WFS
    device-input call refuses it before any launch and the context stays usable."""
    import torch
    from maos_b200 import shwfs
    from maos_b200.configs import LGS8_N32_2WVL
    from maos_b200.workload import build
    wl = build(LGS8_N32_2WVL, device=0, seed=4, noisy=False, nx=512)
    ctx = wl.ctx
    opd = torch.zeros(1 << 16, device="cuda:0")
    llt = torch.zeros(1 << 12, device="cuda:0")
    with pytest.raises(shwfs.ShwfsError, match="frame path"):
        ctx.ints_grad_dev(wl.wfs[0], 0, opd, lltopd=llt)
    wl.frame(2)
    assert all(np.isfinite(g).all() for g in wl.frame_sync())
    wl.close()


@pytest.mark.parametrize("cfg_name,opts,form", [("LGS8_N32_2WVL", {"dtrat": 2}, 0),
                                                ("LGS8_N32_2WVL", {"sigmatch": 2}, 0),
                                                ("NGS8_2WVL", {"sigmatch": 2}, 0),
                                                ("LGS8_N32_2WVL", {}, 1)])
def test_bands_compose_with_integration_and_normalisation(ref_lib, cfg_name, opts, form):
    """Bands under the other imaging layers: dtrat integration sums the band-summed frames of a
    period, sigmatch 2 normalises by the total of the band sum, and the tensor-core form images
    each band of an LGS powfs with that band's uplink; against the reference's own frames of the
    same polychromatic powfs."""
    from maos_b200 import configs
    from maos_b200.workload import build
    from tests.helpers import ints_tolerance_ok, grad_rel_err
    dtrat = opts.get("dtrat", 1)
    cfg = dict(getattr(configs, cfg_name))
    if "sigmatch" in opts:
        cfg.update(name=cfg["name"] + "_sig2", sigmatch=opts["sigmatch"])
    wl = build(cfg, device=0, seed=6, noisy=False, nx=512, form=form)
    if dtrat > 1:
        wl.ctx.powfs_set_dtrat(wl.ipowfs, dtrat)
    r = ref_lib.RefPowfs(cfg)
    if cfg["phytype"] == 1:
        for i in wl.wfs:
            wl.ctx.wfs_set_mtche(i, r.mtche(), r.i0sum(), r.i0sumsum())
    ref_lib.atm_set(wl.screens, wl.layers)
    frames = list(range(4, 4 + dtrat))
    for isim in frames:
        wl.frame(isim)
    out = wl.frame_sync(want_ints=True)
    tol = 1e-4 if form == 1 else 1e-5
    for k in range(len(wl.wfs)):
        ints_ref = sum(ref_lib.frame_full_mt(r, k, isim, cfg["dt"], noisy=False)[0] for isim in frames)
        g, ints = out[k]
        ok, worst = ints_tolerance_ok(ints, ints_ref, r.nsa, r.npix, tol)
        assert ok, f"wfs {k}: intensity error {worst:.3e} of subaperture total"
        g_ref = r.grad(ints_ref, iwfs=k)
        assert grad_rel_err(g, g_ref) <= 1e-4, (k, grad_rel_err(g, g_ref))
    wl.close()
