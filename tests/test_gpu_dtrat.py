"""Integration over dtrat frames (powfs.dtrat): the intensities of the frames
of a period add up, and the last frame forms the gradients of the sum, as the
reference integrates in wfsints and forms gradients on its output frames.
Checked against the sum of the reference's own frames on the same screens
(noise-free; intensities within 1e-5 of the subaperture total, gradients
within 1e-4 relative), in the FFT and tensor-core forms (1e-4 intensities)."""
import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


@pytest.mark.parametrize("form", ["fft", "tc"])
def test_ngs_dtrat3_matches_reference_sum(ref_lib, form):
    from maos_b200 import shwfs
    from maos_b200.configs import NGS8
    from maos_b200.workload import build
    from tests.helpers import ints_tolerance_ok, grad_rel_err
    f = shwfs.SHWFS_FORM_TC if form == "tc" else shwfs.SHWFS_FORM_FFT
    wl = build(NGS8, device=0, seed=2, noisy=False, nx=512, form=f)
    wl.ctx.powfs_set_dtrat(wl.ipowfs, 3)
    r = ref_lib.RefPowfs(NGS8)
    ref_lib.atm_set(wl.screens, wl.layers)
    g_before = None
    ints_sum = 0
    for isim in (3, 4, 5):
        wl.frame(isim)
        g, ints = wl.frame_sync(want_ints=True)[0]
        ints_ref, _, _ = ref_lib.frame_full_mt(r, 0, isim, NGS8["dt"], noisy=False)
        ints_sum = ints_sum + ints_ref
        if isim < 5:
            # no output yet: the gradients stay as they were (zero before any output frame)
            assert not np.any(g)
        ok, worst = ints_tolerance_ok(ints, ints_sum, r.nsa, r.npix, 1e-5 if form == "fft" else 1e-4)
        assert ok, (isim, worst)
    g_ref = r.grad(ints_sum)
    assert grad_rel_err(g, g_ref) <= 1e-4, grad_rel_err(g, g_ref)
    # the next period starts a new sum
    wl.frame(6)
    _, ints6 = wl.frame_sync(want_ints=True)[0]
    ints_ref6, _, _ = ref_lib.frame_full_mt(r, 0, 6, NGS8["dt"], noisy=False)
    ok, worst = ints_tolerance_ok(ints6, ints_ref6, r.nsa, r.npix, 1e-5 if form == "fft" else 1e-4)
    assert ok, worst
    wl.close()


def test_lgs_dtrat2_frame(ref_lib):
    from maos_b200.configs import LGS8_N32
    from maos_b200.workload import build
    from tests.helpers import ints_tolerance_ok, grad_rel_err
    wl = build(LGS8_N32, device=0, seed=5, noisy=False, nx=512)
    wl.ctx.powfs_set_dtrat(wl.ipowfs, 2)
    r = ref_lib.RefPowfs(LGS8_N32)
    for i in wl.wfs:
        wl.ctx.wfs_set_mtche(i, r.mtche(), r.i0sum(), r.i0sumsum())
    ref_lib.atm_set(wl.screens, wl.layers)
    for isim in (8, 9):
        wl.frame(isim)
    out = wl.frame_sync(want_ints=True)
    for k in range(len(wl.wfs)):
        a = ref_lib.frame_full_mt(r, k, 8, LGS8_N32["dt"], noisy=False)[0]
        b = ref_lib.frame_full_mt(r, k, 9, LGS8_N32["dt"], noisy=False)[0]
        g, ints = out[k]
        ok, worst = ints_tolerance_ok(ints, a + b, r.nsa, r.npix, 1e-5)
        assert ok, worst
        assert grad_rel_err(g, r.grad(a + b, iwfs=k)) <= 1e-4
    wl.close()


@pytest.mark.parametrize("cfg_name", ["LGS8_N64", "NGS30_2X2"])
def test_dtrat2_larger_sizes(ref_lib, cfg_name):
    """Integration over 2 frames in the 64-point fused kernel (LGS, matched filter) and in the
    FFT-pass chain's pixel step (the 2x2 NGS at FFT 128, CoG): the intensities of the period
    add up and its last frame forms the gradients of the sum."""
    from maos_b200 import configs
    from maos_b200.workload import build
    from tests.helpers import ints_tolerance_ok, grad_rel_err
    cfg = getattr(configs, cfg_name)
    wl = build(cfg, device=0, seed=5, noisy=False, nx=512)
    wl.ctx.powfs_set_dtrat(wl.ipowfs, 2)
    r = ref_lib.RefPowfs(cfg)
    if cfg["phytype"] == 1:
        for i in wl.wfs:
            wl.ctx.wfs_set_mtche(i, r.mtche(), r.i0sum(), r.i0sumsum())
    ref_lib.atm_set(wl.screens, wl.layers)
    for isim in (12, 13):
        wl.frame(isim)
    out = wl.frame_sync(want_ints=True)
    for k in range(len(wl.wfs)):
        a = ref_lib.frame_full_mt(r, k, 12, cfg["dt"], noisy=False)[0]
        b = ref_lib.frame_full_mt(r, k, 13, cfg["dt"], noisy=False)[0]
        g, ints = out[k]
        ok, worst = ints_tolerance_ok(ints, a + b, r.nsa, r.npix, 1e-5)
        assert ok, worst
        assert grad_rel_err(g, r.grad(a + b, iwfs=k)) <= 1e-4
    wl.close()
