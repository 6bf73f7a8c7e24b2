"""Closed-loop terms of the WFS OPD on the GPU against the reference's CPU frame.

In closed loop MAOS subtracts the deformable mirrors from every WFS OPD and adds
tip/tilt, focus and static surfaces (maos/wfsgrad.c:200-262; the GPU path
cuda/sim/wfsgrad.cu:531-605).  The library takes the mirror grids
(shwfs_dm_set), the per-WFS terms (shwfs_wfs_set_opd_terms) and the NCPA
surface (shwfs_wfs_set_opdadd); the oracle applies the same terms with the
reference's own prop (wrap=0, alpha=-1), loc_add_ptt, loc_add_focus,
loc_add_focus_offset and the uplink tip/tilt on the LLT OPD.

Tolerances as the other frame tests: OPD within 1e-5 of its peak; noise-free
intensities within 1e-5 of the subaperture total; gradients within 1e-4
relative."""
import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def _mirrors(D, seed):
    """Two mirror grids (ground and 9 km) of smooth surfaces, 0.5 m pitch,
    covering every footprint of a D m telescope with margin."""
    rng = np.random.default_rng(seed)
    out, surf = [], []
    for ht, n in ((0.0, int(D / 0.5) + 9), (9000.0, int(D / 0.5) + 15)):
        dx = 0.5
        o = -(n // 2) * dx
        x = o + dx * np.arange(n)
        X, Y = np.meshgrid(x, x)
        s = np.zeros((n, n))
        for _ in range(6):
            kx, ky = rng.uniform(-1.2, 1.2, 2)
            s += rng.normal(0, 1.5e-7) * np.cos(kx * X + ky * Y + rng.uniform(0, 2 * np.pi))
        out.append(dict(nx=n, ny=n, dx=dx, ox=o, oy=o, ht=ht, alpha=-1.0))
        surf.append(s)
    return out, surf


def _terms(cfg, nsa, nopd, seed):
    rng = np.random.default_rng(seed)
    llt = bool(cfg.get("has_llt"))
    return dict(ptt=(2e-8, 1.2e-7, -0.8e-7), focus_tel=4e-9, focus_llt=3e-9 if llt else 0.0,
                lltptt=(2e-7, -1.5e-7) if llt else (0.0, 0.0),
                opdadd=rng.normal(0, 3e-8, nsa * nopd * nopd))


@pytest.mark.parametrize("cfg_name,isim", [("LGS8_N32", 7), ("NGS8", 3), ("LGS8_N64", 5)])
def test_closed_loop_frame_matches_reference(ref_lib, cfg_name, isim):
    import torch
    from maos_b200 import configs
    from maos_b200.workload import build
    from tests.helpers import ints_tolerance_ok, grad_rel_err
    cfg = getattr(configs, cfg_name)
    wl = build(cfg, device=0, seed=4, noisy=False, nx=512)
    r = ref_lib.RefPowfs(cfg)
    if cfg["phytype"] == 1:
        for i in wl.wfs:
            wl.ctx.wfs_set_mtche(i, r.mtche(), r.i0sum(), r.i0sumsum())
    ref_lib.atm_set(wl.screens, wl.layers)
    mir, surf = _mirrors(cfg["D"], seed=9)
    t = _terms(cfg, r.nsa, r.nopd, seed=10)
    ctx = wl.ctx
    ctx.copy_counters()
    ctx.dm_set(mir, surf)
    h2d, _ = ctx.copy_counters()
    assert h2d == 4 * sum(s.size for s in surf)  # the mirror surfaces, FP32
    for i in wl.wfs:
        ctx.wfs_set_opd_terms(i, use_dm=True, ptt=t["ptt"], focus_tel=t["focus_tel"], focus_llt=t["focus_llt"],
                              lltptt=t["lltptt"])
        ctx.wfs_set_opdadd(i, t["opdadd"])
    ref_lib.cl_set(mir, surf, use_dm=True, ptt=t["ptt"], focus_tel=t["focus_tel"], focus_llt=t["focus_llt"],
                   lltptt=t["lltptt"], opdadd=t["opdadd"])
    dev = torch.device("cuda", 0)
    for k in range(len(wl.wfs)):
        opd_ref, _ = ref_lib.frame_opd(r, k, isim, cfg["dt"])
        opd = torch.zeros(r.nsa * r.nopd ** 2, dtype=torch.float32, device=dev)
        ctx.raytrace_dev(wl.wfs[k], isim, opd)
        ctx.sync()
        o = opd.double().cpu().numpy()
        assert np.abs(o - opd_ref).max() <= 1e-5 * np.abs(opd_ref).max(), k
    wl.frame(isim)
    out = wl.frame_sync(want_ints=True)
    for k in range(len(wl.wfs)):
        ints_ref, g_ref, _ = ref_lib.frame_full_mt(r, k, isim, cfg["dt"], noisy=False)
        g, ints = out[k]
        ok, worst = ints_tolerance_ok(ints, ints_ref, r.nsa, r.npix, 1e-5)
        assert ok, f"wfs {k}: intensity error {worst:.3e} of subaperture total"
        assert grad_rel_err(g, g_ref) <= 1e-4, (k, grad_rel_err(g, g_ref))
    # the terms change the gradients: the same frame without them differs
    ref_lib.cl_set()
    _, g_ol, _ = ref_lib.frame_full_mt(r, 0, isim, cfg["dt"], noisy=False)
    assert grad_rel_err(out[0][0], g_ol) > 1e-2
    wl.close()


def test_mirror_points_off_grid_or_nan_add_nothing():
    """A mirror whose surface is NaN everywhere (points outside the actuator
    region, add_valid of math/numtype.h:40), or whose grid lies away from the
    pupil (wrap=0), leaves the OPD as it is, bit for bit; a WFS that does not
    use the mirrors ignores them."""
    import torch
    from maos_b200.configs import NGS8
    from maos_b200.workload import build
    wl = build(NGS8, device=0, seed=4, noisy=False, nx=512)
    ctx, iw = wl.ctx, wl.wfs[0]
    n = wl.nsa * wl.setup.nopd ** 2
    dev = torch.device("cuda", 0)
    base = torch.zeros(n, dtype=torch.float32, device=dev)
    ctx.raytrace_dev(iw, 2, base)
    grids = [dict(nx=30, ny=30, dx=0.5, ox=-7.5, oy=-7.5, ht=0.0, alpha=-1.0),
             dict(nx=10, ny=10, dx=0.5, ox=40.0, oy=40.0, ht=0.0, alpha=-1.0)]
    ctx.dm_set(grids, [np.full((30, 30), np.nan), np.ones((10, 10))])
    for use in (True, False):
        ctx.wfs_set_opd_terms(iw, use_dm=use)
        o = torch.zeros_like(base)
        ctx.raytrace_dev(iw, 2, o)
        ctx.sync()
        assert torch.equal(o, base), use
    # a finite mirror on the pupil changes it
    ctx.dm_set(grids, [np.full((30, 30), 1e-7), np.ones((10, 10))])
    ctx.wfs_set_opd_terms(iw, use_dm=True)
    o = torch.zeros_like(base)
    ctx.raytrace_dev(iw, 2, o)
    ctx.sync()
    d = (o - base).double().cpu().numpy()
    assert np.allclose(d, -1e-7, rtol=0, atol=1e-12)
    wl.close()
