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
