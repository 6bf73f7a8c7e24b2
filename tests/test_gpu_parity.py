"""Parity of the CUDA frame with the reference's own FFTW-double path.

Inputs (pupil, DTF, ETF, pixel map, matched filter, OPD) come from the
reference's setup and ray trace (oracle/_ref); the GPU runs through the C ABI.
Tolerances: noise-free pixel intensities within 1e-5 of the subaperture total,
gradients within 1e-4 relative (max |dg| / max |g_ref|)."""
import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

INTS_REL = 1e-5
GRAD_REL = 1e-4


def _run_gpu(ctx, iwfs, nsa, npix, opd, lltopd=None):
    import torch
    dev = torch.device("cuda", 0)
    o = torch.tensor(opd, dtype=torch.float32, device=dev)
    l = torch.tensor(lltopd, dtype=torch.float32, device=dev) if lltopd is not None else None
    ints = torch.zeros(nsa * npix, dtype=torch.float32, device=dev)
    grad = torch.zeros(2 * nsa, dtype=torch.float32, device=dev)
    ctx.ints_grad_dev(iwfs, 0, o, l, ints, grad)
    ctx.sync()
    return ints.double().cpu().numpy(), grad.double().cpu().numpy()


@pytest.mark.parametrize("seed", [1, 2])
def test_ngs8_cog_parity(ref_lib, seed):
    from maos_b200.configs import NGS8
    from tests.helpers import context_from_ref, turbulent_opd, ints_tolerance_ok, grad_rel_err
    ref = ref_lib.RefPowfs(NGS8)
    opd, _ = turbulent_opd(ref, seed=seed)
    opd32 = opd.astype(np.float32).astype(np.float64)
    ints_ref = ref.wfsints(opd32)
    g_ref = ref.grad(ints_ref)
    ctx, ip, iw = context_from_ref(ref, NGS8)
    ints, g = _run_gpu(ctx, iw[0], ref.nsa, ref.npix, opd32)
    ok, worst = ints_tolerance_ok(ints, ints_ref, ref.nsa, ref.npix, INTS_REL)
    assert ok, f"intensity error {worst:.3e} of subaperture total"
    assert grad_rel_err(g, g_ref) <= GRAD_REL, grad_rel_err(g, g_ref)
    ctx.close()


def test_lgs30_mf_parity(ref_lib):
    from maos_b200.configs import LGS30
    from tests.helpers import context_from_ref, turbulent_opd, ints_tolerance_ok, grad_rel_err
    ref = ref_lib.RefPowfs(LGS30)
    opd, scr = turbulent_opd(ref, seed=3)
    opd32 = opd.astype(np.float32).astype(np.float64)
    n = scr.shape[0]
    ox = -n / 2 / 32.0
    lltopd = ref.prop_llt(scr, 1.0 / 32, ox, ox, 0.0, LGS30["thetax"][0] - LGS30["llt_ox"] / LGS30["hs"],
                          LGS30["thetay"][0] - LGS30["llt_oy"] / LGS30["hs"], LGS30["hs"], LGS30["llt_ox"],
                          LGS30["llt_oy"])
    llt32 = lltopd.astype(np.float32).astype(np.float64)
    ints_ref = ref.wfsints(opd32, llt32)
    g_ref = ref.grad(ints_ref)
    ctx, ip, iw = context_from_ref(ref, LGS30)
    ints, g = _run_gpu(ctx, iw[0], ref.nsa, ref.npix, opd32, llt32)
    ok, worst = ints_tolerance_ok(ints, ints_ref, ref.nsa, ref.npix, INTS_REL)
    assert ok, f"intensity error {worst:.3e} of subaperture total"
    assert grad_rel_err(g, g_ref) <= GRAD_REL, grad_rel_err(g, g_ref)
    ctx.close()
