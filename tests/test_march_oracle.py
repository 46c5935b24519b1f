"""The ray-marching oracle (orc_m_fp_view) against analytic line integrals.

A Gaussian blob f = exp(-r^2 / (2 s^2)) sampled at voxel centres has, along a
line at distance b from its centre, the integral sqrt(2 pi) s exp(-b^2 / (2 s^2)).
GEOMETRIC plane sampling with trilinear interpolation reproduces it to the
interpolation error (s = 6 voxels: well under 1 %).  REFERENCE mode normalises
every axis by (Ydim-1)*YVoxSize, i.e. it projects the volume stretched by
Ydim/(Ydim-1), point sampled: it agrees to a few per cent.
"""
import numpy as np
import pytest

from conftest import rel_l2, small_cfg

from oracle import oracle as O
from recon_b200.configs import geom_dict

N, SIGMA = 48, 6.0


def _case():
    cfg = small_cfg(Xdim=N, Ydim=N, Zdim=N)
    g = O.Geom.from_dict(geom_dict(cfg))
    c = np.arange(N) - (N - 1) / 2
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    vol = np.exp(-(x * x + y * y + z * z) / (2.0 * SIGMA ** 2)).astype(np.float32).ravel()
    return cfg, g, vol


def _analytic(cfg):
    """Line integrals of the continuous blob along each pixel's ray (any view angle)."""
    Nu, Nv, R, Rf = cfg["AxPixels"], cfg["TAxPixels"], cfg["R"], cfg["Rf"]
    du, dv = cfg["AxPixDim"] * cfg["M"], cfg["TAxPixDim"] * cfg["M"]
    u_id = (-(Nu - 1) / 2 + np.arange(Nu)) * du * R / cfg["Ry"]
    v_id = (-(Nv - 1) / 2 + np.arange(Nv)) * dv * R / cfg["Ry"]
    U, V = np.meshgrid(u_id, v_id)
    n2 = U * U + V * V + R * R
    b2 = Rf * Rf * (1.0 - R * R / n2)  # squared distance from the centre to the ray
    s = SIGMA * cfg["XVoxSize"]
    return (np.sqrt(2.0 * np.pi) * s * np.exp(-b2 / (2.0 * s * s))).ravel()


@pytest.mark.parametrize("angle", [0.0, 30.0, 117.0])
def test_geometric_marching_matches_analytic_integrals(angle):
    cfg, g, vol = _case()
    march = O.m_fp_view(g, angle, 1, vol)
    assert rel_l2(march, _analytic(cfg)) < 1e-2, rel_l2(march, _analytic(cfg))


def test_reference_marching_is_a_stretched_line_integral():
    cfg, g, vol = _case()
    march = O.m_fp_view(g, 0.0, 0, vol)
    assert rel_l2(march, _analytic(cfg)) < 0.1, rel_l2(march, _analytic(cfg))
