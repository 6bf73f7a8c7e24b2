"""Tensor-core (tcgen05, BF16x3 split DFT) form against the reference's FP64
FFTW path (oracle/_ref) and against the FP32 FFT form.

Every test reports the errors it measured.  Bars: gradients within 1e-4
relative (max |dg| / max |g|) of FP64, intensities within 1e-4 of the
subaperture total."""
import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

TC_INTS = 1e-4
TC_GRAD = 1e-4


def _run(ctx, iwfs, nsa, npix, opd, lltopd=None):
    import torch
    dev = torch.device("cuda", 0)
    o = torch.tensor(opd, dtype=torch.float32, device=dev)
    l = torch.tensor(lltopd, dtype=torch.float32, device=dev) if lltopd is not None else None
    ints = torch.zeros(nsa * npix, dtype=torch.float32, device=dev)
    grad = torch.zeros(2 * nsa, dtype=torch.float32, device=dev)
    ctx.ints_grad_dev(iwfs, 0, o, l, ints, grad)
    ctx.sync()
    return ints.double().cpu().numpy(), grad.double().cpu().numpy()


def _errors(ints, ints_ref, g, g_ref, nsa, npix):
    from tests.helpers import ints_tolerance_ok, grad_rel_err
    _, wi = ints_tolerance_ok(ints, ints_ref, nsa, npix, 1.0)
    return wi, grad_rel_err(g, g_ref)


@pytest.mark.parametrize("seed", [1, 4])
def test_tc_ngs8_vs_fp64(ref_lib, seed):
    from maos_b200 import shwfs
    from maos_b200.configs import NGS8
    from tests.helpers import context_from_ref, turbulent_opd
    ref = ref_lib.RefPowfs(NGS8)
    opd, _ = turbulent_opd(ref, seed=seed)
    opd = opd.astype(np.float32).astype(np.float64)
    ints_ref = ref.wfsints(opd)
    g_ref = ref.grad(ints_ref)
    ctx, ip, iw = context_from_ref(ref, NGS8)
    ctx.set_form(shwfs.SHWFS_FORM_TC)
    ints, g = _run(ctx, iw[0], ref.nsa, ref.npix, opd)
    wi, wg = _errors(ints, ints_ref, g, g_ref, ref.nsa, ref.npix)
    print(f"TC NGS8 seed {seed}: intensity err {wi:.2e} of subaperture total, gradient err {wg:.2e}")
    assert wi <= TC_INTS and wg <= TC_GRAD
    ctx.close()


def test_tc_lgs30_vs_fp64(ref_lib):
    from maos_b200 import shwfs
    from maos_b200.configs import LGS30
    from tests.helpers import context_from_ref, turbulent_opd
    ref = ref_lib.RefPowfs(LGS30)
    opd, scr = turbulent_opd(ref, seed=3)
    opd = opd.astype(np.float32).astype(np.float64)
    n = scr.shape[0]
    ox = -n / 2 / 32.0
    llt = ref.prop_llt(scr, 1.0 / 32, ox, ox, 0.0, LGS30["thetax"][0] - LGS30["llt_ox"] / LGS30["hs"],
                       LGS30["thetay"][0] - LGS30["llt_oy"] / LGS30["hs"], LGS30["hs"], LGS30["llt_ox"],
                       LGS30["llt_oy"]).astype(np.float32).astype(np.float64)
    ints_ref = ref.wfsints(opd, llt)
    g_ref = ref.grad(ints_ref)
    ctx, ip, iw = context_from_ref(ref, LGS30)
    ctx.set_form(shwfs.SHWFS_FORM_TC)
    ints, g = _run(ctx, iw[0], ref.nsa, ref.npix, opd, llt)
    wi, wg = _errors(ints, ints_ref, g, g_ref, ref.nsa, ref.npix)
    print(f"TC LGS30: intensity err {wi:.2e} of subaperture total, gradient err {wg:.2e}")
    assert wi <= TC_INTS and wg <= TC_GRAD
    ctx.close()


def test_tc_full_frame_matches_fft_form():
    """Whole frames (ray trace, uplink, noise-free imaging, matched filter) of
    the product workload in both forms."""
    from maos_b200 import shwfs
    from maos_b200.configs import LGS30
    from maos_b200.workload import build
    from tests.helpers import ints_tolerance_ok, grad_rel_err
    wl = build(LGS30, device=0, seed=2, noisy=False, nx=512)
    wl.frame(9)
    fft = wl.frame_sync(want_ints=True)
    wl.ctx.set_form(shwfs.SHWFS_FORM_TC)
    wl.frame(9)
    tc = wl.frame_sync(want_ints=True)
    for (gf, inf_), (gt, int_) in zip(fft, tc):
        ok, wi = ints_tolerance_ok(int_, inf_, wl.nsa, wl.npix, TC_INTS)
        assert ok, wi
        assert grad_rel_err(gt, gf) <= TC_GRAD
    wl.close()
