"""Full-frame parity of the larger FFT sizes (the FFT-pass chain) against the
reference's own CPU frame (oracle/_ref) on the same screens: LGS with 32x32
OPD points and FFT 64 (the large-sampling stress sampling, on an 8 m
telescope) and FFT 128 (the same pupils embedded four times), the 2x2 NGS
with FFT 128 and the 1x1 tip-tilt sensors with FFT 256 of the uneven batch.

Tolerances as for the 32-point path: noise-free intensities within 1e-5 of the
subaperture total, gradients within 1e-4 relative (max |dg| / max |g|)."""
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def _check(ref_lib, cfg, isim, use_ref_mtche):
    from maos_b200.workload import build
    from tests.helpers import ints_tolerance_ok, grad_rel_err
    wl = build(cfg, device=0, seed=4, noisy=False, nx=512)
    r = ref_lib.RefPowfs(cfg)
    if use_ref_mtche:
        for i in wl.wfs:
            wl.ctx.wfs_set_mtche(i, r.mtche(), r.i0sum(), r.i0sumsum())
    ref_lib.atm_set(wl.screens, wl.layers)
    wl.frame(isim)
    out = wl.frame_sync(want_ints=True)
    for k in range(len(wl.wfs)):
        ints_ref, g_ref, _ = ref_lib.frame_full_mt(r, k, isim, cfg["dt"], noisy=False)
        g, ints = out[k]
        ok, worst = ints_tolerance_ok(ints, ints_ref, r.nsa, r.npix, 1e-5)
        assert ok, f"{cfg['name']} wfs {k}: intensity error {worst:.3e} of subaperture total"
        assert grad_rel_err(g, g_ref) <= 1e-4, (cfg["name"], k, grad_rel_err(g, g_ref))
    wl.close()


@pytest.mark.parametrize("isim", [0, 29])
def test_lgs_fft64_frame_matches_reference(ref_lib, isim):
    from maos_b200.configs import LGS8_N64
    _check(ref_lib, LGS8_N64, isim, use_ref_mtche=True)


def test_lgs_fft128_frame_matches_reference(ref_lib):
    """An LGS powfs through the FFT-pass chain: 32x32 OPD points embedded four times (FFT
    128), 8x8 pixels of 0.8" -- pass 3's multiply by the elongation transfer function, and the
    uplink OTF formed by passes 1-3 at 128 points."""
    from maos_b200.configs import LGS8_N64
    cfg = dict(LGS8_N64, name="lgs8_2x8x8_n128", embfac=4, notf=128, pixpsa=8)
    _check(ref_lib, cfg, 11, use_ref_mtche=True)


def test_ngs_fft128_frame_matches_reference(ref_lib):
    from maos_b200.configs import NGS30_2X2
    _check(ref_lib, NGS30_2X2, 7, use_ref_mtche=False)


def test_tiptilt_fft256_frame_matches_reference(ref_lib):
    from maos_b200.configs import TT30
    _check(ref_lib, TT30, 3, use_ref_mtche=False)


def test_stress_config_full_size_matches_reference(ref_lib):
    """The large-sampling stress configuration at its full size: 30 m telescope, 6 LGS of
    60x60 subapertures (2820 valid), 32x32 OPD points, FFT 64, 12x12 pixels of 0.8", the
    two-Gaussian sodium profile (88 and 94 km) and 7 layers on 4096^2 screens at 1/64 m.
    The product's own setup and matched filter throughout; two WFS on two frames against the
    reference's CPU frame on the same screens, with its own setup and matched filter."""
    import os
    from maos_b200.configs import LGS30_N64
    from maos_b200.workload import build
    from tests.helpers import ints_tolerance_ok, grad_rel_err
    cfg = LGS30_N64
    wl = build(cfg, device=0, seed=4, noisy=False)
    assert wl.nsa == 2820 and wl.setup.notf == 64 and wl.npix == 144 and wl.screens[0].shape == (4096, 4096)
    r = ref_lib.RefPowfs(cfg, nthread=os.cpu_count() or 1)
    ref_lib.atm_set(wl.screens, wl.layers)
    for isim in (0, 17):
        wl.frame(isim)
        out = wl.frame_sync(want_ints=True)
        for k in (0, 4):
            ints_ref, g_ref, _ = ref_lib.frame_full_mt(r, k, isim, cfg["dt"], noisy=False)
            g, ints = out[k]
            ok, worst = ints_tolerance_ok(ints, ints_ref, r.nsa, r.npix, 1e-5)
            assert ok, f"wfs {k}: intensity error {worst:.3e} of subaperture total"
            assert grad_rel_err(g, g_ref) <= 1e-4, (isim, k, grad_rel_err(g, g_ref))
    wl.close()
