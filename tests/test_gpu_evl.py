"""Science path on the GPU (include/shwfs_evl.h) against the reference's own
open-loop evaluation (oracle/_ref: setup_aper, prop onto aper->locs,
loc_calc_ptt, locfft_psf) on the same screens and aperture.

Tolerances: OPD within 1e-5 of its peak; PR/TT/PTTR variances within 1e-4
relative; mode coefficients within 1e-4 of the largest; the PSF within 2e-5
of its peak (FP32 transforms of up to 1024 points) and its sum within 1e-5."""
import math

import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

AS2RAD = math.pi / 180 / 3600


def _setup(ref_lib, D, Din, dx, wvl, nembed, psfsize, pttr, dirs, seed=7, nx=1024):
    from maos_b200 import shwfs
    from maos_b200.configs import LGS30
    from maos_b200.setup import aperture, screens
    from maos_b200.workload import wind
    x, y, a = aperture(D, Din, dx)
    ctx = shwfs.Context(0)
    ctx.set_dt(1 / 800)
    cfg = dict(LGS30, atm=dict(LGS30["atm"], nx=nx, dx=1 / 32))
    at = cfg["atm"]
    scr = screens(nx, nx, at["dx"], at["r0"], at["L0"], at["wt"], seed)
    vx, vy = wind(cfg, seed)
    o = -nx / 2 * at["dx"]
    layers = [dict(nx=nx, ny=nx, dx=at["dx"], ox=o, oy=o, ht=float(h), vx=float(vx[i]), vy=float(vy[i]), alpha=1.0)
              for i, h in enumerate(at["ht"])]
    ctx.atm_set(layers, scr)
    ref_lib.atm_set(scr, layers)
    ctx.evl_set_aper(x, y, dx, a)
    for d in dirs:
        ctx.evl_add_dir(*d)
    ctx.evl_set_psf(wvl, nembed, psfsize, pttr=pttr)
    e = ref_lib.RefEvl(D, Din, dx, wvl=wvl, nembed=nembed)
    rx, ry, ra = e.aper()
    assert np.array_equal(rx, x) and np.array_equal(ra, a)
    return ctx, e, len(x)


@pytest.mark.parametrize("pttr", [0, 1])
def test_evl_matches_reference(ref_lib, pttr):
    import torch
    wvl, nembed, psfsize = [1.25e-6, 2.2e-6], [512, 1024], [128, 1024]
    dirs = [(0.0, 0.0, math.inf), (20 * AS2RAD, -10 * AS2RAD, math.inf), (5 * AS2RAD, 5 * AS2RAD, 90e3)]
    ctx, e, nloc = _setup(ref_lib, 8.0, 1.2, 1 / 32, wvl, nembed, psfsize, pttr, dirs)
    frames = [3, 11]
    psf_ref = [[np.zeros((n, n)) for n in psfsize] for _ in dirs]
    for isim in frames:
        ctx.evl_queue(isim, do_psf=True)
        wfe, coeff = ctx.evl_sync()
        for k, (tx, ty, hs) in enumerate(dirs):
            opd_r, wfe_r, coeff_r, psf_r = e.frame(tx, ty, hs, isim, 1 / 800, pttr=pttr, psfsize=psfsize)
            opd = torch.zeros(nloc, dtype=torch.float32, device="cuda")
            ctx.evl_opd_dev(k, opd)
            ctx.sync()
            o = opd.double().cpu().numpy()
            assert np.abs(o - opd_r).max() <= 1e-5 * np.abs(opd_r).max(), (isim, k)
            assert np.all(np.abs(wfe[k] - wfe_r) <= 1e-4 * np.abs(wfe_r)), (isim, k, wfe[k], wfe_r)
            assert np.abs(coeff[k] - coeff_r).max() <= 1e-4 * np.abs(coeff_r).max(), (isim, k)
            for w in range(len(wvl)):
                psf_ref[k][w] += psf_r[w]
    for k in range(len(dirs)):
        for w in range(len(wvl)):
            p, nf = ctx.evl_psf(k, w)
            r = psf_ref[k][w]
            assert nf == len(frames)
            assert np.abs(p - r).max() <= 2e-5 * r.max(), (k, w, np.abs(p - r).max() / r.max())
            assert abs(p.sum() - r.sum()) <= 1e-5 * r.sum()
    ctx.evl_psf_reset()
    p, nf = ctx.evl_psf(0, 0)
    assert nf == 0 and not p.any()
    ctx.close()


def test_evl_rejects_bad_sizes(ref_lib):
    from maos_b200 import shwfs
    from maos_b200.setup import aperture
    x, y, a = aperture(4.0, 0.5, 1 / 16)
    ctx = shwfs.Context(0)
    ctx.evl_set_aper(x, y, 1 / 16, a)
    for bad in ([300], [32], [8192]):
        with pytest.raises(shwfs.ShwfsError):
            ctx.evl_set_psf([1e-6], bad)
    with pytest.raises(shwfs.ShwfsError):
        ctx.evl_set_psf([1e-6], [64])  # 65 points do not fit a 64-point grid
    with pytest.raises(shwfs.ShwfsError):
        ctx.evl_set_psf([1e-6], [256], [255])
    with pytest.raises(shwfs.ShwfsError):
        ctx.evl_set_aper(x + 0.3 * (1 / 16) * (np.arange(len(x)) % 2), y, 1 / 16, a)  # off the grid
    ctx.close()
