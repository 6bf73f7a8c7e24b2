"""The autotuner times whole frames of every imaging-kernel variant on the
device and keeps the fastest; the frames it leaves behind are the frames of
the variant it chose, bit for bit."""
import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def test_autotune_keeps_a_variant_and_its_frames():
    from maos_b200.configs import LGS8_N32
    from maos_b200.workload import build
    wl = build(LGS8_N32, device=0, seed=3, noisy=True, nx=256)
    v = wl.ctx.autotune(wl.wfs[0], wl.wfs[-1] + 1, nrep=2)
    assert 0 <= v < 6  # SHWFS_NVARIANT
    wl.frame(1)
    a = wl.frame_sync(want_ints=True)
    wl.ctx.set_variant(wl.ipowfs, v)
    wl.frame(1)
    b = wl.frame_sync(want_ints=True)
    for (ga, ia), (gb, ib) in zip(a, b):
        assert np.isfinite(ga).all() and np.array_equal(ga, gb) and np.array_equal(ia, ib)
    wl.close()
