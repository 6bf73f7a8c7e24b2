"""The product's host setup producers against the reference's own setup
(maos/powfs.c, lib/mkdtf.c, lib/mkh.c, lib/turbulence.c run via oracle/_ref).
Geometry, valid-subaperture selection, pixel maps, DTF, ETF, LLT pupil and
screens are compared bit for bit."""
import numpy as np
import pytest

from maos_b200.configs import NGS8, LGS30, LGS8_N64, NGS30_2X2, TT30, NGS8_2WVL, LGS8_N32_2WVL


def _setup(cfg):
    from maos_b200.setup import Setup
    return Setup(cfg)


@pytest.mark.parametrize("cfg", [NGS8, LGS30, LGS8_N64, NGS30_2X2, TT30], ids=lambda c: c["name"])
def test_geometry_bit_exact(ref_lib, cfg):
    r = ref_lib.RefPowfs(cfg)
    s = _setup(cfg)
    assert s.nsa == r.nsa and s.notf == r.notf and s.nopd == r.nopd
    rx, ry = r.saloc()
    assert np.array_equal(rx, s.get("salocx")) and np.array_equal(ry, s.get("salocy"))
    ox, oy = r.ptsorig()
    assert np.array_equal(ox, s.get("origx")) and np.array_equal(oy, s.get("origy"))
    assert np.array_equal(r.amp(), s.get("amp"))
    assert np.array_equal(r.saa(), s.get("saa"))
    assert s.saasum == r.saasum()  # powfs.saasum, summed as the reference does


@pytest.mark.parametrize("cfg", [NGS8, LGS30, LGS8_N64, NGS30_2X2, TT30], ids=lambda c: c["name"])
def test_dtf_and_pixel_map_bit_exact(ref_lib, cfg):
    from oracle.ref import si_to_taps
    r = ref_lib.RefPowfs(cfg)
    s = _setup(cfg)
    assert np.array_equal(r.nominal(0), s.get("nominal"))
    ri, rw = si_to_taps(r.si_dense(0))
    si = s.simap_idx().reshape(-1, 4)
    sw = s.get("simap_wt").reshape(-1, 4)
    for p in range(len(ri)):
        a = {int(k): v for k, v in zip(ri[p], rw[p]) if k >= 0}
        b = {int(k): v for k, v in zip(si[p], sw[p]) if k >= 0}
        assert a == b, (p, a, b)


@pytest.mark.parametrize("cfg", [NGS8_2WVL, LGS8_N32_2WVL], ids=lambda c: c["name"])
def test_wavelength_bands_bit_exact(ref_lib, cfg):
    """A polychromatic powfs: the product's setup at each band's wavelength gives the
    reference's DTF nominal, pixel map and ETF of that wavelength (powfs.dtf[iwvl],
    etfsim[iwvl]) bit for bit, with the OTF size of the first wavelength."""
    from oracle.ref import si_to_taps
    r = ref_lib.RefPowfs(cfg)
    for iw, wv in enumerate(cfg["wvls"]):
        r.select_wvl(iw)
        s = _setup(dict(cfg, wvl=wv))
        assert s.notf == r.notf and s.nsa == r.nsa
        assert s.dtheta == r.dtheta
        if cfg.get("has_llt"):
            assert np.array_equal(r.etf(), s.get("etf")), iw
        else:
            assert np.array_equal(r.nominal(0), s.get("nominal")), iw
        ri, rw = si_to_taps(r.si_dense(0))
        si = s.simap_idx().reshape(-1, 4)
        sw = s.get("simap_wt").reshape(-1, 4)
        for p in range(len(ri)):
            a = {int(k): v for k, v in zip(ri[p], rw[p]) if k >= 0}
            b = {int(k): v for k, v in zip(si[p], sw[p]) if k >= 0}
            assert a == b, (iw, p, a, b)
        s.close()
    # the two wavelengths sample differently
    r.select_wvl(0)
    d0 = r.dtheta
    r.select_wvl(1)
    assert r.dtheta > d0


def test_lgs_etf_llt_bit_exact(ref_lib):
    r = ref_lib.RefPowfs(LGS30)
    s = _setup(LGS30)
    assert np.array_equal(r.srot(), s.get("srot"))
    assert np.array_equal(r.srsa(), s.get("srsa"))
    assert np.array_equal(r.etf(), s.get("etf"))
    assert np.array_equal(r.lltamp(), s.get("lltamp"))


def test_screen_generator_bit_exact_and_kat(ref_lib):
    from maos_b200.setup import screens
    a = ref_lib.genatm_simple(0.186, 0, -11.0 / 3.0, 1.0 / 64, 128, 1)
    b = screens(128, 128, 1.0 / 64, 0.186, 0, [1.0], 1)[0]
    assert np.array_equal(a, b)
    # test/cmocka_psd.c:49: rms 169.648 nm
    assert abs(np.sqrt((b ** 2).mean()) * 1e9 - 169.648) < 1e-3


def test_seven_layer_screens_bit_exact(ref_lib):
    """The 7-layer atmosphere of the LGS configs against the reference's own
    genscreen (lib/turbulence.c:214) from the same seed: every layer equal."""
    from maos_b200.configs import LGS30
    from maos_b200.setup import screens
    a = LGS30["atm"]
    ref = ref_lib.genscreen(128, 128, a["dx"], a["r0"], a["L0"], a["wt"], 3)
    own = screens(128, 128, a["dx"], a["r0"], a["L0"], a["wt"], 3)
    assert len(ref) == len(own) == 7
    for x, y in zip(ref, own):
        assert np.array_equal(x, y)


def test_two_layer_screens_pairing(ref_lib):
    """Layers come in pairs from one complex transform (real, imaginary)."""
    from maos_b200.setup import screens
    s2 = screens(64, 64, 1.0 / 32, 0.186, 30.0, [0.7, 0.3], 5)
    s1 = screens(64, 64, 1.0 / 32, 0.186, 30.0, [0.7], 5)
    assert np.array_equal(s2[0], s1[0])
    assert abs(np.std(s2[0]) / np.std(s2[1]) - np.sqrt(0.7 / 0.3)) < 0.5


@pytest.mark.parametrize("cfg_name", ["LGS8_N32", "LGS30", "NGS8_MF"])
def test_matched_filter_matches_reference(ref_lib, cfg_name):
    """The product's matched-filter chain against the reference's setup_shwfs_phygrad:
    the short-exposure PSF of every subaperture (genseotf with piston/tip/tilt removed and
    the uplink OTF, gensepsf), i0, gx, gy (gensei), i0sum and mtche (mtch).  They agree to
    about 2e-7 relative: the reference's Bessel function (math/bessik.c) converges to about
    3e-10 relative, and the covariance difference B(0) - B(r) that the OTF exponentiates
    magnifies that by the ratio of the phase variance to the structure function; the
    product's K_5/6 is exact to 1e-15 (checked against scipy)."""
    from maos_b200 import configs
    cfg = dict(configs.NGS8, name="ngs8_16x16_mf", phytype=1) if cfg_name == "NGS8_MF" else getattr(configs, cfg_name)
    r = ref_lib.RefPowfs(cfg)
    s = _setup(cfg)
    n2 = r.notf ** 2
    sp = s.get("sepsf").reshape(r.nsa, n2)
    i0, gx, gy = (s.get(k).reshape(r.nsa, r.npix) for k in ("i0", "gx", "gy"))
    step = max(1, r.nsa // 64)
    for isa in range(0, r.nsa, step):
        ps = r.sepsf(isa)
        assert np.abs(sp[isa] - ps).max() <= 1e-6 * max(np.abs(ps).max(), 1e-300), isa
        ri0, rgx, rgy = r.i0(isa)
        for a, b in ((i0[isa], ri0), (gx[isa], rgx), (gy[isa], rgy)):
            assert np.abs(a - b).max() <= 1e-6 * max(np.abs(b).max(), 1e-300), isa
    assert np.abs(s.get("i0sum") - r.i0sum()).max() <= 1e-6 * r.i0sum().max()
    m, mr = s.get("mtche").reshape(r.nsa, 2 * r.npix), r.mtche()
    assert np.abs(m - mr).max() <= 1e-6 * np.abs(mr).max()
    # the same subapertures are rejected (dim or noisy: rows of zeros)
    assert np.array_equal(np.abs(m).sum(1) == 0, np.abs(mr).sum(1) == 0)
