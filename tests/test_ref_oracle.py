"""The reference's own C code, compiled here as the oracle, reproduces the
known-answer values of its test suite (test/cmocka_psd.c:25-57)."""
import numpy as np
import pytest


def test_screen_kat_matches_reference_test_suite(ref_lib):
    # genatm_simple(0.186, 0, -11/3, 1/64, 128, seed 1): RMS, PSD integrals,
    # fitted r0/slope and structure function, tolerance 1e-3 as in the reference test.
    got = ref_lib.kat_psd()
    want = [169.648, 56.4647, 216.578, 0.128266, -3.68282, 3.01473, 1.15708]
    assert np.allclose(got, want, atol=1e-3, rtol=0), (got, want)


def test_reference_setup_ngs8(ref_lib):
    from maos_b200.configs import NGS8
    ref = ref_lib.RefPowfs(NGS8)
    assert ref.nsa == 204
    assert (ref.notf, ref.nopd, ref.pixpsax) == (32, 16, 8)
    # every pixel of the sampling map has at most 4 taps (bilinear)
    from oracle.ref import si_to_taps
    idx, wt = si_to_taps(ref.si_dense(0))
    assert idx.shape == (64, 4)


def test_reference_setup_lgs30(ref_lib):
    from maos_b200.configs import LGS30
    ref = ref_lib.RefPowfs(LGS30)
    assert ref.nsa == 2820
    assert ref.llt_nx == 16
    m = ref.mtche()
    assert m.shape == (2820, 72) and np.isfinite(m).all()


def _tilt_opd(r, a, b):
    """OPD a x + b y + c over every subaperture's points (nsa nopd^2, x fastest)."""
    ox, oy = r.ptsorig()
    dx = r.ptsdx()
    i = np.arange(r.nopd)
    x = ox[:, None, None] + dx * i[None, None, :]
    y = oy[:, None, None] + dx * i[None, :, None]
    return (a * x + b * y + 3e-7 + 0 * x).ravel()


def test_reference_ztilt_known_answer(ref_lib):
    """pts_ztilt of a plane recovers its slope in every lit subaperture and
    ignores piston (the weighted least-squares fit is exact for a plane)."""
    from maos_b200.configs import NGS8
    r = ref_lib.RefPowfs(NGS8)
    a, b = 2.5e-6, -1.25e-6
    g = r.ztilt(_tilt_opd(r, a, b))
    assert np.allclose(g[:r.nsa], a, rtol=1e-9, atol=0)
    assert np.allclose(g[r.nsa:], b, rtol=1e-9, atol=0)


def test_reference_gtilt_known_answer(ref_lib):
    """GS0 (mkg) applied to a plane gives its slope in every subaperture."""
    from maos_b200.configs import NGS8
    r = ref_lib.RefPowfs(NGS8)
    nrow, ncol, pp, pi, px = r.gs0()
    assert (nrow, ncol) == (2 * r.nsa, r.nsa * r.nopd ** 2) and pp[-1] == len(px)
    a, b = 2.5e-6, -1.25e-6
    g = r.gtilt(_tilt_opd(r, a, b))
    assert np.allclose(g[:r.nsa], a, rtol=1e-9, atol=0)
    assert np.allclose(g[r.nsa:], b, rtol=1e-9, atol=0)


def test_reference_second_etf(ref_lib):
    """The second ETF slot: same focus gives the first ETF, another focus a different one."""
    from maos_b200.configs import LGS30
    r = ref_lib.RefPowfs(LGS30)
    e1 = r.etf()
    r.setup_etf2(0.0, 4)
    assert np.array_equal(r.etf2(), e1)
    r.setup_etf2(2000.0, 4)
    e2 = r.etf2()
    assert np.abs(e2 - e1).max() > 1e-3 * np.abs(e1).max()
