"""Gradient options against the reference's own shwfs_grad (maos/utils.c:
983-1122, dcog math/matmath.c:717-758) on the same noise-free frame:
thresholded CoG with offsets and the three sigmatch normalisations (2: by the
frame's total intensity over all subapertures, summed on the device before
the gradients), and the matched filter with sigmatch 0, 1, 2 and the
cross-coupling options of its construction (mtchcr).

Tolerances as in the frame parity tests: intensities within 1e-5 of the
subaperture total, gradients within 1e-4 relative."""
import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def _check(ref_lib, cfg, seed=4):
    import torch
    from tests.helpers import context_from_ref, turbulent_opd, ints_tolerance_ok, grad_rel_err
    ref = ref_lib.RefPowfs(cfg)
    opd, _ = turbulent_opd(ref, seed=seed)
    opd32 = opd.astype(np.float32).astype(np.float64)
    ints_ref = ref.wfsints(opd32)
    g_ref = ref.grad(ints_ref)
    ctx, ip, iw = context_from_ref(ref, cfg)
    dev = torch.device("cuda", 0)
    o = torch.tensor(opd32, dtype=torch.float32, device=dev)
    ints = torch.zeros(ref.nsa * ref.npix, dtype=torch.float32, device=dev)
    g = torch.zeros(2 * ref.nsa, dtype=torch.float32, device=dev)
    ctx.ints_grad_dev(iw[0], 0, o, None, ints, g)
    # the same gradients from the stored intensities (shwfs_grad_dev)
    g2 = torch.zeros(2 * ref.nsa, dtype=torch.float32, device=dev)
    ctx.grad_dev(iw[0], ints, g2)
    ctx.sync()
    ok, worst = ints_tolerance_ok(ints.double().cpu().numpy(), ints_ref, ref.nsa, ref.npix, 1e-5)
    assert ok, worst
    e = grad_rel_err(g.double().cpu().numpy(), g_ref)
    assert e <= 1e-4, (cfg["name"], e)
    assert np.array_equal(g.cpu().numpy(), g2.cpu().numpy())
    ctx.close()


@pytest.mark.parametrize("sigmatch,cogthres,cogoff", [(0, 0.0, 0.0), (1, 0.0, 0.0), (2, 0.0, 0.0), (1, 20.0, 0.0),
                                                      (1, 0.0, 5.0), (2, 10.0, 3.0), (0, 15.0, 2.0)])
def test_cog_options_match_reference(ref_lib, sigmatch, cogthres, cogoff):
    from maos_b200.configs import NGS8
    cfg = dict(NGS8, name=f"ngs8_cog_s{sigmatch}_t{cogthres}_o{cogoff}", sigmatch=sigmatch, cogthres=cogthres,
               cogoff=cogoff)
    _check(ref_lib, cfg)


@pytest.mark.parametrize("sigmatch,mtchcr", [(0, 0), (1, 0), (2, 0), (1, 1), (2, 1)])
def test_mf_options_match_reference(ref_lib, sigmatch, mtchcr):
    from maos_b200.configs import NGS8
    cfg = dict(NGS8, name=f"ngs8_mf_s{sigmatch}_c{mtchcr}", phytype=1, sigmatch=sigmatch, mtchcr=mtchcr)
    _check(ref_lib, cfg)


@pytest.mark.parametrize("cfg_name,form", [("LGS8_N32", "fft"), ("LGS8_N64", "fft"), ("NGS30_2X2", "fft"),
                                           ("LGS8_N32", "tc")])
def test_lgs_sigmatch2_frame_matches_reference(ref_lib, cfg_name, form):
    """A whole frame (ray trace, uplink, imaging, device sum, gradients) with sigmatch 2
    against the reference's frame: LGS at FFT 32 (FFT and tensor-core forms) and 64 (matched
    filter), the 2x2 NGS at FFT 128 (CoG)."""
    from maos_b200 import configs, shwfs
    from maos_b200.workload import build
    from tests.helpers import ints_tolerance_ok, grad_rel_err
    base = getattr(configs, cfg_name)
    cfg = dict(base, name=base["name"] + "_sig2", sigmatch=2)
    f = shwfs.SHWFS_FORM_TC if form == "tc" else shwfs.SHWFS_FORM_FFT
    wl = build(cfg, device=0, seed=3, noisy=False, nx=512, form=f)
    r = ref_lib.RefPowfs(cfg)
    if cfg["phytype"] == 1:
        for i in wl.wfs:
            wl.ctx.wfs_set_mtche(i, r.mtche(), r.i0sum(), r.i0sumsum())
    ref_lib.atm_set(wl.screens, wl.layers)
    wl.frame(6)
    out = wl.frame_sync(want_ints=True)
    for k in range(len(wl.wfs)):
        ints_ref, g_ref, _ = ref_lib.frame_full_mt(r, k, 6, cfg["dt"], noisy=False)
        g, ints = out[k]
        ok, worst = ints_tolerance_ok(ints, ints_ref, r.nsa, r.npix, 1e-4 if form == "tc" else 1e-5)
        assert ok, worst
        assert grad_rel_err(g, g_ref) <= 1e-4, (k, grad_rel_err(g, g_ref))
    wl.close()
