"""Science aperture (CPU): the product's standalone aperture builder
(shwfs_aper_build) is bit-exact with the reference's setup_aper for an
annulus (create_metapupil, loc_from_map, mkamp, loc_reduce, normalisation),
and the reference's open-loop evaluation obeys its defining identities on a
planar OPD (the oracle's own check)."""
import math

import numpy as np
import pytest


@pytest.mark.parametrize("D,Din,dx", [(4.0, 0.5, 1 / 16), (8.0, 1.2, 1 / 32), (30.0, 3.6, 1 / 32)])
def test_aperture_bit_exact(ref_lib, D, Din, dx):
    from maos_b200.setup import aperture
    x, y, a = aperture(D, Din, dx)
    e = ref_lib.RefEvl(D, Din, dx)
    rx, ry, ra = e.aper()
    assert len(x) == len(rx)
    assert np.array_equal(x, rx) and np.array_equal(y, ry) and np.array_equal(a, ra)


def test_reference_evl_plane(ref_lib):
    e = ref_lib.RefEvl(4.0, 0.5, 1 / 16, wvl=[1.65e-6], nembed=[256])
    n, dx = 512, 1 / 32
    yy, xx = np.mgrid[0:n, 0:n] * dx - n / 2 * dx
    scr = 1e-6 * (0.3 * xx - 0.2 * yy) + 2e-7
    ref_lib.atm_set([scr], [dict(nx=n, ny=n, dx=dx, ox=-n / 2 * dx, oy=-n / 2 * dx, ht=0.0, vx=0.0, vy=0.0)])
    opd, wfe, coeff, psf = e.frame(0, 0, math.inf, 0, 1 / 800, pttr=1, psfsize=[64])
    assert np.allclose(coeff, [2e-7, 3e-7, -2e-7], rtol=1e-9)
    assert abs(wfe[2]) < 1e-20 and wfe[0] > 0 and abs(wfe[0] - wfe[1]) < 1e-20
    assert abs(psf[0].max() - 1.0) < 1e-9  # flat wavefront after tip/tilt removal: (sum amp)^2
