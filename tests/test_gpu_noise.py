"""Photon and read noise on the GPU (shwfs_addnoise_dev, the rule of addnoise
in lib/libmisc.c:31-55) against exact distributions.

The Poisson sampler of the frame kernels switches method at a mean of 10
(inversion below, transformed rejection up to 200) and uses the reference's
Gaussian rule above 200.  For means on both sides of each switch, 4e5 draws
are binned and compared with the Poisson pmf by a chi-square test (bins with
fewer than 20 expected counts are pooled); the extended rule (excess factor,
quantum efficiency, per-pixel backgrounds, read noise) is checked through its
mean and variance."""
import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

N = 400_000


def _ctx():
    from maos_b200 import shwfs
    return shwfs.Context(device=0)


def _draw(ctx, lam, seed=7, frame=0, **kw):
    import torch
    x = torch.full((N,), float(lam), dtype=torch.float32, device="cuda")
    ctx.addnoise_dev(x, seed=seed, frame=frame, **kw)
    ctx.sync()
    return x.double().cpu().numpy()


def _chi2_poisson(v, lam):
    from scipy import stats
    k = np.rint(v).astype(np.int64)
    assert np.all(k >= 0) and np.allclose(v, k)
    lo, hi = int(stats.poisson.ppf(1e-9, lam)), int(stats.poisson.isf(1e-9, lam)) + 1
    edges = np.arange(lo, hi + 1)
    pmf = stats.poisson.pmf(edges[:-1], lam)
    pmf[0] += stats.poisson.cdf(lo - 1, lam)
    pmf[-1] += stats.poisson.sf(hi - 1, lam)
    obs = np.bincount(np.clip(k, lo, hi - 1) - lo, minlength=hi - lo).astype(float)
    exp = pmf * len(k)
    # pool bins with small expectation into their neighbours
    o2, e2, ao, ae = [], [], 0.0, 0.0
    for a, b in zip(obs, exp):
        ao += a
        ae += b
        if ae >= 20:
            o2.append(ao)
            e2.append(ae)
            ao = ae = 0.0
    if ae > 0:
        o2[-1] += ao
        e2[-1] += ae
    o2, e2 = np.array(o2), np.array(e2)
    e2 *= o2.sum() / e2.sum()
    return stats.chisquare(o2, e2).pvalue


@pytest.mark.parametrize("lam", [0.05, 0.7, 3.3, 9.99, 10.0, 17.5, 64.0, 150.0, 199.9])
def test_poisson_matches_pmf(lam):
    ctx = _ctx()
    v = _draw(ctx, lam)
    p = _chi2_poisson(v, lam)
    assert p > 1e-4, (lam, p)
    # mean and variance within 6 standard errors
    assert abs(v.mean() - lam) <= 6 * np.sqrt(lam / N)
    assert abs(v.var() - lam) <= 6 * lam * np.sqrt(2.0 / N) + 6 * np.sqrt(lam / N)
    ctx.close()


def test_gaussian_rule_above_200():
    ctx = _ctx()
    lam = 350.0
    v = _draw(ctx, lam)
    assert np.allclose(v, np.rint(v))
    assert abs(v.mean() - lam) <= 6 * np.sqrt(lam / N)
    assert abs(v.var() / lam - 1) <= 6 * np.sqrt(2.0 / N) + 1e-3
    ctx.close()


def test_counter_based_and_deterministic():
    ctx = _ctx()
    a = _draw(ctx, 12.0, seed=3, frame=5)
    b = _draw(ctx, 12.0, seed=3, frame=5)
    c = _draw(ctx, 12.0, seed=3, frame=6)
    assert np.array_equal(a, b)
    assert np.mean(a != c) > 0.5
    ctx.close()


def test_extended_rule_moments():
    """x = (P(tot e) + tot (1-e) + rne N) qe - corr with tot = (x + b + b2) qe."""
    import torch
    ctx = _ctx()
    rng = np.random.default_rng(1)
    npix = 64
    x0 = rng.uniform(0.0, 40.0, npix)
    b2 = rng.uniform(0.0, 3.0, npix)
    b2c = rng.uniform(0.0, 1.0, npix)
    qe = rng.uniform(0.7, 1.2, npix)
    bk, bkc, rne, ex = 1.5, 0.5, 2.5, 1.4
    reps = N // npix
    dev = "cuda"
    x = torch.tensor(np.tile(x0, reps), dtype=torch.float32, device=dev)
    t = lambda a: torch.tensor(np.tile(a, reps), dtype=torch.float32, device=dev)
    ctx.addnoise_dev(x, seed=11, bkgrnd=bk, bkgrndc=bkc, rne=rne, excess=ex, bkgrnd2=t(b2), bkgrnd2c=t(b2c), qe=t(qe))
    ctx.sync()
    v = x.double().cpu().numpy().reshape(reps, npix)
    tot = (x0 + bk + b2) * qe
    mean = tot * qe - (bkc + b2c)
    var = (tot * ex + rne ** 2) * qe ** 2
    m, s2 = v.mean(0), v.var(0)
    assert np.all(np.abs(m - mean) <= 6 * np.sqrt(var / reps))
    assert np.all(np.abs(s2 - var) <= 6 * var * np.sqrt(2.0 / reps) + 6 * np.sqrt(var / reps))
    ctx.close()
