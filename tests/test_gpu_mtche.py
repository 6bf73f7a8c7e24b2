"""Matched filter regenerated on the device (shwfs_wfs_update_mtche) against the
reference's own (setup_shwfs_phygrad: genseotf, gensepsf, gensei, mtch).

The device forms i0, gx and gy from the short-exposure OTF that the host setup
uploads (shwfs_powfs_set_seotf: turbulence with piston/tip/tilt removed times
the conjugate uplink OTF, as genseotf/gensepsf build it) times the current
ETF or DTF nominal, then inverts as lib/mtch.c does.  Bars: the matched filter
within 1e-4 of its largest element, i0 sums within 1e-4 of their largest, the
same subapertures rejected, and the gradients of a noise-free frame through
the device filter within 1e-4 relative of the reference's CPU frame; and the
device filter against the host-built one through the same frame."""
import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def _cfg(name):
    from maos_b200 import configs
    if name == "NGS8_MF":
        return dict(configs.NGS8, name="ngs8_16x16_mf", phytype=1, mtchcr=0)
    return getattr(configs, name)


@pytest.mark.parametrize("cfg_name,isim,wfs", [("LGS30", 5, (0, 3)), ("LGS8_N32", 9, (0, 1)), ("NGS8_MF", 4, (0,))])
def test_device_matched_filter_matches_reference(ref_lib, cfg_name, isim, wfs):
    from maos_b200.workload import build
    from tests.helpers import grad_rel_err
    cfg = _cfg(cfg_name)
    wl = build(cfg, device=0, seed=8, noisy=False, nx=512)
    r = ref_lib.RefPowfs(cfg)
    for i in wl.wfs:
        wl.ctx.wfs_update_mtche(i, cfg["mtchcr"])
    mr, sr = r.mtche(), r.i0sum()
    for i in wl.wfs:
        m, s, tot = wl.ctx.wfs_get_mtche(i)
        assert np.abs(m - mr).max() <= 1e-4 * np.abs(mr).max(), (i, np.abs(m - mr).max() / np.abs(mr).max())
        assert np.abs(s - sr).max() <= 1e-4 * sr.max()
        assert abs(tot - r.i0sumsum()) <= 1e-4 * r.i0sumsum()
        assert np.array_equal(np.abs(m).sum(1) == 0, np.abs(mr).sum(1) == 0)
    ref_lib.atm_set(wl.screens, wl.layers)
    wl.frame(isim)
    g = wl.frame_sync()
    for k in wfs:
        _, g_ref, _ = ref_lib.frame_full_mt(r, k, isim, cfg["dt"], noisy=False)
        assert grad_rel_err(g[k], g_ref) <= 1e-4, (k, grad_rel_err(g[k], g_ref))
    wl.close()


@pytest.mark.parametrize("cfg_name", ["LGS30", "NGS8_MF"])
def test_device_matched_filter_matches_host_setup(cfg_name):
    """The device-regenerated filter and the host setup's give the same gradients of one
    noise-free frame within 1e-4 relative."""
    from maos_b200.workload import build
    from tests.helpers import grad_rel_err
    cfg = _cfg(cfg_name)
    wl = build(cfg, device=0, seed=8, noisy=False, nx=512)
    wl.frame(5)
    g_host = wl.frame_sync()
    for i in wl.wfs:
        wl.ctx.wfs_update_mtche(i, cfg["mtchcr"])
    wl.frame(5)
    g_dev = wl.frame_sync()
    wl.close()
    for a, b in zip(g_dev, g_host):
        assert abs(b).max() > 0
        assert grad_rel_err(a, b) <= 1e-4, grad_rel_err(a, b)
