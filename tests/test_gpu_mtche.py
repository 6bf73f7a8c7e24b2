"""Matched filter regenerated on the device (shwfs_wfs_update_mtche) against
the host-built one (the project's setup, lib/gensei.c + lib/mtch.c rules):
the gradients of the same noise-free frame agree within 1e-4 relative, for
the LGS sensors (ETF, flat uplink OTF, cross-coupling terms) and for an NGS
matched filter (DTF nominal, no cross-coupling)."""
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def _compare(cfg, mtchcr):
    from maos_b200.workload import build
    from tests.helpers import grad_rel_err
    wl = build(cfg, device=0, seed=8, noisy=False, nx=512)
    wl.frame(5)
    g_host = wl.frame_sync()
    for i in wl.wfs:
        wl.ctx.wfs_update_mtche(i, mtchcr)
    wl.frame(5)
    g_dev = wl.frame_sync()
    wl.close()
    for a, b in zip(g_dev, g_host):
        assert abs(b).max() > 0
        assert grad_rel_err(a, b) <= 1e-4, grad_rel_err(a, b)


def test_lgs_matched_filter_regenerated_on_device():
    from maos_b200.configs import LGS30
    _compare(LGS30, LGS30["mtchcr"])


def test_ngs_matched_filter_regenerated_on_device():
    from maos_b200.configs import NGS8
    _compare(dict(NGS8, name="ngs8_16x16_mf", phytype=1, mtchcr=0), 0)
