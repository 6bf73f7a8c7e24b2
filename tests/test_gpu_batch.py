"""The uneven batch (LGS FFT 32, NGS FFT 128, tip-tilt FFT 256 on one
atmosphere) through the CUDA-graph frame: identical to the plain stream
frame, bit for bit, over several frames (the graph carries each frame's
parameters), and each sensor type matches its own single-powfs frame."""
import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def _frames(graph, isims, noisy, worklist=False, slices=0, priority=True):
    from maos_b200.configs import UNEVEN_BATCH
    from maos_b200.workload import build_batch
    wl = build_batch(UNEVEN_BATCH["members"], device=0, seed=6, noisy=noisy, nx=512, graph=graph)
    if not priority:
        wl.ctx.set_branch_priority(False)
    if worklist:
        wl.ctx.set_worklist(True, slices)
    out = []
    for isim in isims:
        wl.frame(isim)
        out.append(wl.frame_sync(want_ints=True))
    wl.close()
    return out


@pytest.mark.parametrize("noisy", [False, True])
def test_graph_frames_equal_stream_frames(noisy):
    isims = [0, 1, 2, 5, 9]
    a = _frames(False, isims, noisy)
    b = _frames(True, isims, noisy)
    for fa, fb in zip(a, b):
        for (ga, ia), (gb, ib) in zip(fa, fb):
            assert np.array_equal(ga, gb) and np.array_equal(ia, ib)
    # the frames differ from each other (wind, noise counters)
    assert not np.array_equal(a[0][0][0], a[-1][0][0])


def test_batch_members_match_single_powfs_frames():
    from maos_b200.configs import UNEVEN_BATCH, NGS30_2X2, TT30
    from maos_b200.workload import build
    b = _frames(True, [0, 3], False)[-1]
    # NGS (index 6) and tip-tilt (7, 8) on the same screens, alone
    for cfg, idx in ((NGS30_2X2, [6]), (TT30, [7, 8])):
        wl = build(dict(cfg, atm=UNEVEN_BATCH["members"][0]["atm"]), device=0, seed=6, noisy=False, nx=512)
        wl.frame(3)
        single = wl.frame_sync(want_ints=True)
        wl.close()
        for k, j in enumerate(idx):
            assert np.array_equal(single[k][0], b[j][0]) and np.array_equal(single[k][1], b[j][1])


def test_range_sync_equals_per_wfs_sync():
    """One range sync of the whole batch frame returns every WFS's gradients
    as the per-WFS syncs do."""
    from maos_b200.configs import UNEVEN_BATCH
    from maos_b200.workload import build_batch
    wl = build_batch(UNEVEN_BATCH["members"], device=0, seed=6, noisy=True, nx=512, graph=True)
    wl.frame(4)
    a = wl.frame_sync()                      # one range call
    wl.frame(4)
    b = [g for g, _ in wl.frame_sync(want_ints=True)]  # per-WFS calls
    wl.close()
    assert len(a) == len(b) == 9
    for ga, gb in zip(a, b):
        assert np.array_equal(ga, gb)


def test_range_sync_into_caller_buffer():
    """The range sync into a caller-owned buffer writes the same gradients as
    the per-WFS arrays, in WFS order, and refuses a buffer that is too small
    or not float64."""
    import pytest
    from maos_b200.configs import UNEVEN_BATCH
    from maos_b200.workload import build_batch
    wl = build_batch(UNEVEN_BATCH["members"], device=0, seed=6, noisy=True, nx=512, graph=True)
    wl.frame(4)
    a = wl.frame_sync()
    n = sum(len(g) for g in a)
    buf = np.full(n, np.nan)
    wl.frame(4)
    assert wl.frame_sync(out=buf) is buf
    assert np.array_equal(buf, np.concatenate(a))
    with pytest.raises(ValueError):
        wl.frame_sync(out=np.empty(n - 1))
    with pytest.raises(ValueError):
        wl.frame_sync(out=np.empty(n, dtype=np.float32))
    wl.close()


@pytest.mark.parametrize("graph,slices", [(False, 8), (True, 8), (True, 3)])
def test_worklist_frames_equal_branch_frames(graph, slices):
    """The frame's imaging as one persistent work-list launch (32-point groups,
    pass tiles of the 128- and 256-point images waiting on their previous pass,
    pixel steps) gives the frames of the per-powfs launches, bit for bit, as a
    stream frame and as a CUDA graph, with the passes interleaved at two slice
    counts; noisy frames, so the noise counters are exercised too."""
    isims = [0, 1, 4, 7]
    a = _frames(False, isims, True)
    b = _frames(graph, isims, True, worklist=True, slices=slices)
    for fa, fb in zip(a, b):
        for (ga, ia), (gb, ib) in zip(fa, fb):
            assert np.isfinite(ga).all()
            assert np.array_equal(ga, gb) and np.array_equal(ia, ib)


def test_worklist_single_powfs_frames_equal():
    """A frame of one 32-point powfs through the work list equals the ordinary launch."""
    from maos_b200.configs import LGS8_N32
    from maos_b200.workload import build
    out = []
    for wlon in (False, True):
        wl = build(LGS8_N32, device=0, seed=2, noisy=True, nx=512)
        wl.ctx.set_variant(wl.ipowfs, 1)
        wl.ctx.set_worklist(wlon)
        wl.frame(3)
        out.append(wl.frame_sync(want_ints=True))
        wl.close()
    for (ga, ia), (gb, ib) in zip(*out):
        assert np.array_equal(ga, gb) and np.array_equal(ia, ib)



def test_frame_layout_autotuner_keeps_a_layout_and_its_frames():
    """shwfs_autotune_frame times the per-powfs launches and the work list at its settings and
    keeps one; the frames after it are the frames of every layout, bit for bit."""
    from maos_b200.configs import UNEVEN_BATCH
    from maos_b200.workload import build_batch
    ref = _frames(False, [3], True)[0]
    wl = build_batch(UNEVEN_BATCH["members"], device=0, seed=6, noisy=True, nx=512, graph=True)
    c = wl.ctx.autotune_frame(0, wl.nwfs, nrep=2)
    assert 0 <= c <= 4
    wl.frame(3)
    out = wl.frame_sync(want_ints=True)
    wl.close()
    for (ga, ia), (gb, ib) in zip(ref, out):
        assert np.array_equal(ga, gb) and np.array_equal(ia, ib)


@pytest.mark.parametrize("graph", [False, True])
def test_branch_priority_keeps_frames(graph):
    """The smaller powfs' branches at the greatest stream priority change the order in which
    blocks reach the SMs, not the frames: identical, bit for bit, with and without."""
    isims = [2, 7]
    a = _frames(graph, isims, True, priority=True)
    b = _frames(graph, isims, True, priority=False)
    for fa, fb in zip(a, b):
        for (ga, ia), (gb, ib) in zip(fa, fb):
            assert np.array_equal(ga, gb) and np.array_equal(ia, ib)


def test_tc_form_frames_in_the_batch_graph():
    """The tensor-core form of the 32-point LGS powfs (its imaging kernel and the separate
    noise/gradient kernel) on a graph branch beside the FFT-pass chains of the NGS and tip-tilt
    sensors: noisy graph frames equal stream frames, bit for bit, and are finite."""
    from maos_b200 import shwfs
    from maos_b200.configs import UNEVEN_BATCH
    from maos_b200.workload import build_batch
    outs = []
    for graph in (False, True):
        wl = build_batch(UNEVEN_BATCH["members"], device=0, seed=6, noisy=True, nx=512, graph=graph,
                         form=shwfs.SHWFS_FORM_TC)
        frames = []
        for isim in (2, 3, 4):
            wl.frame(isim)
            frames.append(wl.frame_sync(want_ints=True))
        wl.close()
        outs.append(frames)
    for fa, fb in zip(*outs):
        for (ga, ia), (gb, ib) in zip(fa, fb):
            assert np.array_equal(ga, gb) and np.array_equal(ia, ib)
            assert np.isfinite(ga).all() and np.isfinite(ia).all()
