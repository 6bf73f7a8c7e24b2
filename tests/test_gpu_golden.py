"""The CUDA path against the committed golden fixtures (tests/golden/), with no
oracle at run time: the product's own setup (bit-exact with the reference's)
loads a context, the fixture's OPD (and LLT OPD) goes through the C ABI
(shwfs_ints_grad_dev: uplink, field, PSF, OTF x transfer functions, pixels,
gradients), and the result is compared with the reference's intensities and
gradients.  Geometric gradients: shwfs_grad_ztilt_dev and a G-tilt sensor
with the fixture's GS0.

Tolerances: noise-free intensities within 1e-5 of the subaperture total
(1e-4 for the BF16x3 tensor-core form), gradients within 1e-4 relative
(max |dg| / max |g|); geometric gradients within 1e-5 relative."""
import numpy as np
import pytest

from tests.conftest import cuda_available
from tests.test_golden import golden, meta

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def _run(case, form, variant=None):
    import torch
    from maos_b200 import shwfs
    from maos_b200.configs import CONFIGS
    from maos_b200.workload import build
    from tests.helpers import ints_tolerance_ok, grad_rel_err
    m = meta(case)
    cfg = CONFIGS[m["config"]]
    iwfs, isim = int(m["iwfs"]), int(m["isim"])
    wl = build(cfg, device=0, seed=1, noisy=False, nx=256, form=form)
    nsa, npix = wl.setup.nsa, wl.setup.npix
    iw = wl.wfs[iwfs]
    if variant is not None:
        wl.ctx.set_variant(wl.ipowfs, variant)
    if cfg["phytype"] == 1:
        mt = golden(case, "mtche")
        mtche = np.stack([mt[i, 0].ravel() for i in range(nsa)])
        i0sum, kw = golden(case, "i0sum", keywords=True)
        wl.ctx.wfs_set_mtche(iw, mtche, i0sum.ravel(), float(kw.split("=")[1]))
    opd = torch.from_numpy(golden(case, "opd").ravel().copy()).cuda()
    llt = None
    if cfg.get("has_llt"):
        llt = torch.from_numpy(golden(case, "lltopd").ravel().copy()).cuda()
    ints = torch.zeros(nsa * npix, dtype=torch.float32, device="cuda")
    grad = torch.zeros(2 * nsa, dtype=torch.float32, device="cuda")
    wl.ctx.ints_grad_dev(iw, isim, opd, llt, ints, grad)
    wl.ctx.sync()
    ints_ref = golden(case, "ints").ravel(order="F")
    g_ref = golden(case, "grad").ravel()
    tol = 1e-4 if form == shwfs.SHWFS_FORM_TC else 1e-5
    ok, worst = ints_tolerance_ok(ints.double().cpu().numpy(), ints_ref, nsa, npix, tol)
    assert ok, f"{case}: intensity error {worst:.3e} of subaperture total"
    e = grad_rel_err(grad.double().cpu().numpy(), g_ref)
    assert e <= 1e-4, (case, e)
    wl.close()


@pytest.mark.parametrize("case", ["ngs8", "lgs8_n32", "lgs8_n64"])
def test_fft_form_matches_golden(case):
    from maos_b200 import shwfs
    _run(case, shwfs.SHWFS_FORM_FFT)


@pytest.mark.parametrize("case", ["ngs8", "lgs8_n32"])
@pytest.mark.parametrize("variant", [1, 2, 3, 4, 5])
def test_fft_form_variants_match_golden(case, variant):
    """Every imaging-kernel variant of the 32-point FFT form (register caps of the full-spectrum
    transforms; the half-spectrum form) against the same fixtures."""
    from maos_b200 import shwfs
    _run(case, shwfs.SHWFS_FORM_FFT, variant)


@pytest.mark.parametrize("case", ["ngs8", "lgs8_n32"])
def test_tc_form_matches_golden(case):
    from maos_b200 import shwfs
    _run(case, shwfs.SHWFS_FORM_TC)


def test_geometric_gradients_match_golden():
    import torch
    from maos_b200 import shwfs
    from maos_b200.configs import NGS8
    from maos_b200.setup import Setup
    s = Setup(NGS8)
    nsa = s.nsa
    ctx = shwfs.Context(0)
    ip = ctx.powfs_add(nsa=nsa, nopd=s.nopd, embfac=1, notf=0, pixpsax=0, pixpsay=0, dsa=NGS8["dsa"], dx=s.dx,
                       hs=NGS8["hs"], areascale=1.0, wvl=NGS8["wvl"], gradtype=shwfs.SHWFS_GRAD_GTILT)
    ctx.powfs_set_geom(ip, s.get("origx"), s.get("origy"), s.get("amp"))
    g0 = golden("ngs8", "gs0")
    ctx.powfs_set_gs0(ip, g0.shape[0], g0.shape[1], g0.indptr, g0.indices, g0.data)
    iw = ctx.wfs_add(ipowfs=ip, thetax=0.0, thetay=0.0, hs=NGS8["hs"], hc=0.0, misregx=0.0, misregy=0.0, sigsim=1.0,
                     wvlwt=1.0, noisy=0)
    opd = torch.from_numpy(golden("ngs8", "opd").ravel().copy()).cuda()
    gz = torch.zeros(2 * nsa, dtype=torch.float32, device="cuda")
    gg = torch.zeros(2 * nsa, dtype=torch.float32, device="cuda")
    ctx.grad_ztilt_dev(iw, opd, gz)
    ctx.grad_gtilt_dev(iw, opd, gg)
    ctx.sync()
    for got, what in ((gz, "ztilt"), (gg, "gtilt")):
        ref = golden("ngs8", what).ravel()
        e = np.abs(got.double().cpu().numpy() - ref).max() / np.abs(ref).max()
        assert e <= 1e-5, (what, e)
    ctx.close()
    s.close()


def test_science_path_matches_golden():
    """The science path on the fixture's aperture (the product's builder,
    bit-exact with the reference's) and screens (the product's generator,
    bit-exact too): OPD within 1e-5 of its peak, PR/TT/PTTR within 1e-4
    relative, the PSF within 2e-5 of its peak."""
    import math
    import torch
    from maos_b200 import shwfs
    from maos_b200.configs import CONFIGS
    from maos_b200.setup import aperture, screens
    from maos_b200.workload import wind
    from tests.test_golden import evl_meta
    m = evl_meta()
    D, Din, dx = float(m["D"]), float(m["Din"]), float(m["dx"])
    cfg = CONFIGS[m["screen_config"]]
    nx, seed = int(m["screen_nx"]), int(m["screen_seed"])
    at = cfg["atm"]
    scr = screens(nx, nx, at["dx"], at["r0"], at["L0"], at["wt"], seed)
    vx, vy = wind(cfg, seed)
    o = -nx / 2 * at["dx"]
    layers = [dict(nx=nx, ny=nx, dx=at["dx"], ox=o, oy=o, ht=float(h), vx=float(vx[i]), vy=float(vy[i]), alpha=1.0)
              for i, h in enumerate(at["ht"])]
    x, y, a = aperture(D, Din, dx)
    ctx = shwfs.Context(0)
    ctx.set_dt(cfg["dt"])
    ctx.atm_set(layers, scr)
    ctx.evl_set_aper(x, y, dx, a)
    ndir = int(m["ndir"])
    for k in range(ndir):
        _, kw = golden(f"evl4_dir{k}", "opd", keywords=True)
        d = dict(line.split("=", 1) for line in kw.splitlines())
        ctx.evl_add_dir(float(d["thetax"]), float(d["thetay"]), float(d["hs"]))
    ctx.evl_set_psf([float(m["wvl"])], [int(m["nembed"])], [int(m["psfsize"])], pttr=int(m["pttr"]))
    ctx.evl_queue(int(m["isim"]), do_psf=True)
    wfe, coeff = ctx.evl_sync()
    for k in range(ndir):
        opd = torch.zeros(len(x), dtype=torch.float32, device="cuda")
        ctx.evl_opd_dev(k, opd)
        ctx.sync()
        o_ref = golden(f"evl4_dir{k}", "opd").ravel()
        assert np.abs(opd.double().cpu().numpy() - o_ref).max() <= 1e-5 * np.abs(o_ref).max()
        w_ref = golden(f"evl4_dir{k}", "wfe").ravel()
        assert np.all(np.abs(wfe[k] - w_ref[:3]) <= 1e-4 * np.abs(w_ref[:3])), (k, wfe[k], w_ref[:3])
        p, nf = ctx.evl_psf(k, 0)
        p_ref = golden(f"evl4_dir{k}", "psf")
        assert nf == 1 and np.abs(p - p_ref).max() <= 2e-5 * p_ref.max()
    ctx.close()
