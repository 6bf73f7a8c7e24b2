"""Serving loop on the GPU: every request's gradients and intensities are the
same, bit for bit, when its simulation is served alone and when the requests
of several simulations are in flight together (each simulation keeps its own
context, stream and noise counters; the kernels are deterministic)."""
import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def _serve(cfgs, arrivals, priority=None):
    from maos_b200.serving import Server
    srv = Server(cfgs, device=0, seed=5, priority=priority)
    srv.prewarm()
    res = {}
    st = srv.run(arrivals, rate=0.0, results=res)
    srv.close()
    assert len(st.latencies_ms) == len(arrivals)
    return res


def test_results_alone_equal_results_in_the_mix():
    from maos_b200.serving import draw_sim_cfg
    cfgs = [draw_sim_cfg(s, screen_nx=256) for s in (3, 11, 21)]  # FFT 64, 32, 32; 2, 4, 1 WFS
    nf = 4
    alone = _serve(cfgs, [(0.0, 0)] * nf)
    mix = _serve(cfgs, [(0.0, k % 3) for k in range(3 * nf)])
    for k in range(nf):
        a, b = alone[(0, k)], mix[(0, k)]
        assert len(a) == len(b) == cfgs[0]["nwfs"]
        for ga, gb in zip(a, b):  # gradients of each WFS
            assert np.array_equal(ga, gb)
    # frames of one simulation differ from one another (wind shift, noise counters)
    assert not np.array_equal(alone[(0, 0)][0], alone[(0, 1)][0])
    assert all((i, k) in mix for i in range(3) for k in range(nf))


@pytest.mark.parametrize("priority", ["large", "small"])
def test_stream_priorities_keep_results(priority):
    """Contexts on streams of different priorities (shwfs_set_stream_priority) serve the same
    gradients, bit for bit, as contexts at the default priority."""
    from maos_b200.serving import draw_sim_cfg
    cfgs = [draw_sim_cfg(s, screen_nx=256) for s in (3, 11, 21)]
    arr = [(0.0, k % 3) for k in range(6)]
    a = _serve(cfgs, arr)
    b = _serve(cfgs, arr, priority=priority)
    assert a.keys() == b.keys()
    for key in a:
        for ga, gb in zip(a[key], b[key]):
            assert np.array_equal(ga, gb)


def test_stream_priority_makes_a_new_stream():
    from maos_b200 import configs
    from maos_b200.workload import build
    import torch
    wl = build(configs.NGS8, device=0, seed=3, noisy=True, nx=256)
    wl.frame(2)
    g0 = wl.frame_sync()
    s0 = wl.ctx.stream
    lo, hi = torch.cuda.Stream.priority_range()
    wl.ctx.set_stream_priority(hi - 10)  # clamped to the greatest priority
    assert wl.ctx.stream != s0
    wl.frame(2)
    g1 = wl.frame_sync()
    wl.close()
    for a, b in zip(g0, g1):
        assert np.array_equal(a, b)
