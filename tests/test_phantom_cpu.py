"""Known answers of the oracle's analytic projectors (the checkers of the GPU projectors).

A sphere of radius R and attenuation mu centred on the isocentre has the line integral 2 R mu
along every ray through its centre; an isotropic Gaussian blob a exp(-r^2 / (2 sigma^2)) has
a sigma sqrt(2 pi). With an odd number of detector columns (and rows) centred at (n - 1) / 2,
the central pixel's ray passes through the isocentre in all seven geometries. For the parallel
kinds a centred blob projects identically in every view.
"""
import math

import numpy as np
import pytest

from cases import KINDS, make_case
from oracle import oracle as orc


def _centre(case):
    return case.og.nr // 2, case.og.nc // 2


@pytest.mark.parametrize("kind", KINDS)
def test_sphere_central_ray(kind):
    case = make_case(kind, nv=12, nc=97, nr=25)
    R, mu = 20.0, 0.02
    p = orc.phantom(case.og, [(0.0, 0.0, 0.0, R, R, R, 0.3, mu)])
    r, c = _centre(case)
    np.testing.assert_allclose(p[:, r, c], 2 * R * mu, rtol=1e-12)
    assert (p >= 0).all() and p.max() <= 2 * R * mu * (1 + 1e-12)


@pytest.mark.parametrize("kind", KINDS)
def test_gaussian_blob_central_ray(kind):
    case = make_case(kind, nv=12, nc=97, nr=25)
    sigma, a = 6.0, 0.03
    p = orc.gauss_project(case.og, [(0.0, 0.0, 0.0, sigma, a)])
    r, c = _centre(case)
    np.testing.assert_allclose(p[:, r, c], a * sigma * math.sqrt(2 * math.pi), rtol=1e-10)
    assert p.max() <= a * sigma * math.sqrt(2 * math.pi) * (1 + 1e-10)


@pytest.mark.parametrize("kind", ["parallel_1d", "parallel_2d"])
def test_centred_blob_is_the_same_in_every_parallel_view(kind):
    case = make_case(kind, nv=16, nc=96, nr=24)
    p = orc.gauss_project(case.og, [(0.0, 0.0, 0.0, 7.0, 0.02)])
    np.testing.assert_allclose(p, np.broadcast_to(p[:1], p.shape), rtol=1e-10, atol=1e-14)


def test_gauss_volume_samples_the_density():
    vol = orc.Volume(8, 6, 4, 1.0, 1.0, 2.0, (0.5, -0.5, 1.0))
    v = orc.gauss_volume(vol, [(1.0, 0.0, 2.0, 3.0, 0.5)])
    # voxel (i, j, k) = (4, 3, 2): x = 0.5 - 3.5 + 4 = 1.0, y = -0.5 - 2.5 + 3 = 0, z = 1 - 3 + 4 = 2
    assert v.shape == (4, 6, 8)
    np.testing.assert_allclose(v[2, 3, 4], 0.5)
    np.testing.assert_allclose(v[0, 0, 0], 0.5 * math.exp(-((-3.0 - 1.0) ** 2 + (-3.0) ** 2 + (-2.0 - 2.0) ** 2) / 18.0))
