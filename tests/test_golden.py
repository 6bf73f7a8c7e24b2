"""The committed golden fixtures (tests/golden/, written by the reference's own
code and .bin writer through tests/golden/make_golden.py):

- they parse with the product's .bin reader, with the shapes and types the
  reference wrote;
- the reference built here reproduces them bit for bit (the oracle pinned
  to the committed vectors);
- the z-tilt and G-tilt gradients obey their defining identities against a
  numpy restatement on the product's own setup geometry (which is bit-exact
  with the reference's).
"""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def golden(case, what, keywords=False):
    from maos_b200.binio import read_bin
    p = os.path.join(GOLDEN, f"{case}_{what}.bin")
    if not os.path.exists(p):
        p += ".gz"
    return read_bin(p, keywords=keywords)


def meta(case):
    _, kw = golden(case, "opd", keywords=True)
    return dict(line.split("=", 1) for line in kw.splitlines())


CASES = ["ngs8", "lgs8_n32", "lgs8_n64"]


@pytest.mark.parametrize("case", CASES)
def test_fixtures_parse(case):
    from maos_b200.configs import CONFIGS
    m = meta(case)
    cfg = CONFIGS[m["config"]]
    opd = golden(case, "opd")
    ints = golden(case, "ints")
    grad = golden(case, "grad")
    assert opd.dtype == np.float32 and opd.shape[1] == 1
    npix, nsa = ints.shape
    assert npix == cfg["pixpsa"] ** 2 and grad.shape == (2 * nsa, 1)
    assert opd.shape[0] % nsa == 0
    assert (ints >= -1e-9 * ints.max()).all() and np.isfinite(grad).all()
    if cfg["phytype"] == 1:
        mt = golden(case, "mtche")
        assert mt.shape == (nsa, 1) and mt[0, 0].shape == (2 * npix, 1)
        _, kw = golden(case, "i0sum", keywords=True)
        assert float(kw.split("=")[1]) > 0


@pytest.mark.parametrize("case", CASES)
def test_reference_reproduces_fixtures(ref_lib, case):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    name, cfg, iwfs, isim, nx, seed = next(c for c in mg.CASES if c[0] == case)
    r = ref_lib.RefPowfs(cfg)
    scr, lay = mg.layers_of(cfg, nx, seed)
    opd, llt = mg.trace(r, cfg, iwfs, isim, scr, lay)
    assert np.array_equal(opd.astype(np.float32), golden(case, "opd").ravel())
    o64 = golden(case, "opd").ravel().astype(np.float64)
    l64 = golden(case, "lltopd").ravel().astype(np.float64) if llt is not None else None
    ints = r.wfsints(o64, l64, iwfs=iwfs, isim=isim)
    assert np.array_equal(ints, golden(case, "ints").ravel(order="F"))
    assert np.array_equal(r.grad(ints, iwfs=iwfs), golden(case, "grad").ravel())


def _ztilt_numpy(opd, ox, oy, dx, amp, nopd):
    """pts_mcc_ptt + inverse + pts_ztilt (math/loc.c:612-650, 839-885) restated."""
    nsa = len(ox)
    o = opd.reshape(nsa, nopd, nopd)
    a = amp.reshape(nsa, nopd, nopd)
    i = np.arange(nopd)
    x = ox[:, None, None] + dx * i[None, None, :]
    y = oy[:, None, None] + dx * i[None, :, None]
    one = np.ones_like(x)
    basis = [one, x, y]
    M = np.array([[np.sum(a * p * q, axis=(1, 2)) for q in basis] for p in basis])  # 3 x 3 x nsa
    b = np.array([np.sum(a * o * p, axis=(1, 2)) for p in basis])  # 3 x nsa
    c = np.linalg.solve(np.moveaxis(M, 2, 0), b.T[:, :, None])[:, :, 0]
    return np.concatenate([c[:, 1], c[:, 2]])


def test_ztilt_fixture_matches_numpy_restatement():
    from maos_b200.configs import NGS8
    from maos_b200.setup import Setup
    s = Setup(NGS8)
    opd = golden("ngs8", "opd").ravel().astype(np.float64)
    g = _ztilt_numpy(opd, s.get("origx"), s.get("origy"), s.dx, s.get("amp"), s.nopd)
    gz = golden("ngs8", "ztilt").ravel()
    assert np.abs(g - gz).max() <= 1e-9 * np.abs(gz).max()
    s.close()


def test_gtilt_fixture_is_gs0_times_opd():
    gs0 = golden("ngs8", "gs0")
    opd = golden("ngs8", "opd").ravel().astype(np.float64)
    gg = golden("ngs8", "gtilt").ravel()
    assert np.abs(gs0 @ opd - gg).max() <= 1e-12 * np.abs(gg).max()


def evl_meta():
    _, kw = golden("evl4_dir0", "opd", keywords=True)
    return dict(line.split("=", 1) for line in kw.splitlines())


def test_evl_fixtures_reproduced_by_reference(ref_lib):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    c = mg.EVL_CASE
    scr, lay = mg.layers_of(c["cfg"], c["nx"], c["seed"])
    ref_lib.atm_set(scr, lay)
    e = ref_lib.RefEvl(c["D"], c["Din"], c["dx"], wvl=c["wvl"], nembed=c["nembed"])
    for k, (tx, ty, hs) in enumerate(c["dirs"]):
        opd, wfe, coeff, psf = e.frame(tx, ty, hs, c["isim"], c["cfg"]["dt"], pttr=c["pttr"], psfsize=c["psfsize"])
        assert np.array_equal(opd, golden(f"evl4_dir{k}", "opd").ravel())
        assert np.array_equal(np.concatenate([wfe, coeff]), golden(f"evl4_dir{k}", "wfe").ravel())
        assert np.array_equal(psf[0], golden(f"evl4_dir{k}", "psf"))
