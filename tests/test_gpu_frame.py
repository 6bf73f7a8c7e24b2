"""Full-frame parity on the GPU: ray trace + uplink + imaging + gradients from
turbulence screens, against the reference's own CPU frame (oracle/_ref) on the
same screens; and statistical parity of the photon/read noise.

Tolerances: OPD within 1e-5 of its peak; noise-free intensities within 1e-5 of
the subaperture total; gradients within 1e-4 relative (max |dg| / max |g|).
Noise: per-pixel mean and variance over 10^4 frames, and a two-sample KS test
against the reference's addnoise (lib/libmisc.c:31) on the same intensities."""
import ctypes

import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def _workload(cfg, noisy=False, nx=512, seed=3):
    from maos_b200.workload import build
    return build(cfg, device=0, seed=seed, noisy=noisy, nx=nx)


@pytest.mark.parametrize("isim", [0, 1000])
def test_raytrace_matches_reference_prop(ref_lib, isim):
    import torch
    from maos_b200.configs import LGS30
    wl = _workload(LGS30)
    r = ref_lib.RefPowfs(LGS30)
    iw = 2  # an off-axis LGS
    opd_ref = np.zeros(r.nsa * r.nopd ** 2)
    dt = LGS30["dt"]
    for L, scr in zip(wl.layers, wl.screens):
        r.prop_layer(scr, L["dx"], L["ox"], L["oy"], L["ht"], LGS30["thetax"][iw], LGS30["thetay"][iw],
                     LGS30["hs"], -L["vx"] * dt * isim, -L["vy"] * dt * isim, opd=opd_ref)
    opd = torch.zeros(r.nsa * r.nopd ** 2, dtype=torch.float32, device="cuda")
    wl.ctx.raytrace_dev(wl.wfs[iw], isim, opd)
    wl.ctx.sync()
    g = opd.double().cpu().numpy()
    assert np.abs(g - opd_ref).max() <= 1e-5 * np.abs(opd_ref).max()
    wl.close()


# imaging variants: 0 full-spectrum transforms, 3 the half-spectrum form
@pytest.mark.parametrize("isim,variant", [(0, 0), (37, 0), (0, 3), (37, 5)])
def test_lgs_full_frame_matches_reference(ref_lib, isim, variant):
    from maos_b200.configs import LGS30
    from tests.helpers import ints_tolerance_ok, grad_rel_err
    wl = _workload(LGS30)
    wl.ctx.set_variant(wl.ipowfs, variant)
    r = ref_lib.RefPowfs(LGS30)
    # same matched filter on both sides (the reference's, built from its turbulence OTF)
    for i in wl.wfs:
        wl.ctx.wfs_set_mtche(i, r.mtche(), r.i0sum(), r.i0sumsum())
    ref_lib.atm_set(wl.screens, wl.layers)
    wl.frame(isim)
    out = wl.frame_sync(want_ints=True)
    for k in (0, 3):
        ints_ref, g_ref, _ = ref_lib.frame_full_mt(r, k, isim, LGS30["dt"], noisy=False)
        g, ints = out[k]
        ok, worst = ints_tolerance_ok(ints, ints_ref, r.nsa, r.npix, 1e-5)
        assert ok, f"wfs {k}: intensity error {worst:.3e} of subaperture total"
        assert grad_rel_err(g, g_ref) <= 1e-4, (k, grad_rel_err(g, g_ref))
    wl.close()


@pytest.mark.parametrize("variant", [0, 3])
def test_ngs_full_frame_matches_reference(ref_lib, variant):
    from maos_b200.configs import NGS8
    from tests.helpers import ints_tolerance_ok, grad_rel_err
    wl = _workload(NGS8)
    wl.ctx.set_variant(wl.ipowfs, variant)
    r = ref_lib.RefPowfs(NGS8)
    ref_lib.atm_set(wl.screens, wl.layers)
    wl.frame(5)
    g, ints = wl.frame_sync(want_ints=True)[0]
    ints_ref, g_ref, _ = ref_lib.frame_full_mt(r, 0, 5, NGS8["dt"], noisy=False)
    ok, worst = ints_tolerance_ok(ints, ints_ref, r.nsa, r.npix, 1e-5)
    assert ok, worst
    assert grad_rel_err(g, g_ref) <= 1e-4
    wl.close()


@pytest.mark.parametrize("variant", [0, 4])
def test_noise_statistics_match_reference(ref_lib, variant):
    """10^4 noisy frames: per-pixel mean and variance, and the distribution of
    normalised residuals against the reference's addnoise on the same image;
    full-spectrum (variant 0) and half-spectrum (variant 4) imaging."""
    from maos_b200.configs import NGS8
    _noise_statistics(ref_lib, NGS8, variant)


def test_noise_statistics_fft128_match_reference(ref_lib):
    """The same statistics for the FFT-pass chain's pixel step (a thread per pixel): the 2x2
    NGS at FFT 128, 256 pixels per subaperture, most of them in the wings (the inversion and
    PTRS rules) and the core above 200 photons (the Gaussian rule)."""
    from maos_b200.configs import NGS30_2X2
    _noise_statistics(ref_lib, NGS30_2X2, None)


def _noise_statistics(ref_lib, cfg, variant):
    import torch
    from scipy import stats
    from tests.helpers import context_from_ref, turbulent_opd
    r = ref_lib.RefPowfs(cfg)
    opd, _ = turbulent_opd(r, seed=11)
    ctx, ip, iw = context_from_ref(r, cfg, noisy=1)
    if variant is not None:
        ctx.set_variant(ip, variant)
    dev = torch.device("cuda", 0)
    o = torch.tensor(opd, dtype=torch.float32, device=dev)
    nf = torch.zeros(r.nsa * r.npix, dtype=torch.float32, device=dev)
    ctx.ints_grad_dev(iw[0], 0, o, None, nf, None, add_noise=False)
    ints = torch.zeros_like(nf)
    s1 = torch.zeros_like(nf, dtype=torch.float64)
    s2 = torch.zeros_like(nf, dtype=torch.float64)
    nframe = 10000
    for k in range(nframe):
        ctx.ints_grad_dev(iw[0], k, o, None, ints, None, add_noise=True)
        d = (ints - nf).double()
        s1 += d
        s2 += d * d
    ctx.sync()
    I = nf.double().cpu().numpy()
    mean = (s1 / nframe).cpu().numpy()
    var = (s2 / nframe).cpu().numpy() - mean ** 2
    rne = cfg["rne"]
    expect_var = I + rne ** 2
    # mean of the residual: 0 within 6 sigma of the mean estimate
    assert np.all(np.abs(mean) <= 6 * np.sqrt(expect_var / nframe) + 1e-3)
    # variance within 6 sigma of the variance estimate (Gaussian approximation, 4th moment ~ 3 var^2 + I)
    sd_var = np.sqrt((2 * expect_var ** 2 + I) / nframe)
    assert np.all(np.abs(var - expect_var) <= 6 * sd_var + 1e-2)
    # distribution: last noisy frame of every pixel vs the reference's addnoise on the same image
    gpu_last = ((ints - nf).double().cpu().numpy()) / np.sqrt(expect_var)
    ref_frames = []
    for seed in range(1, 6):
        x = I.copy()
        ref_lib.lib().oref_addnoise(x.ctypes.data_as(ctypes.c_void_p), ctypes.c_long(len(x)), ctypes.c_uint(seed),
                                    ctypes.c_double(0.0), ctypes.c_double(0.0), ctypes.c_double(rne))
        ref_frames.append((x - I) / np.sqrt(expect_var))
    ref_res = np.concatenate(ref_frames)
    ks = stats.ks_2samp(gpu_last, ref_res)
    assert ks.pvalue > 1e-3, ks
    ctx.close()
