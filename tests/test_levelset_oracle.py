"""The level-set oracle (curvature from psi, DCCD filter, properties) against
the reference's own outputs (tests/golden/levelset_golden.npz, written by
tests/golden/make_golden.py)."""

import os

import numpy as np
import pytest

from oracle import levelset as ol

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "levelset_golden.npz"))


@pytest.mark.parametrize("name", ["f_wall2d", "f_pw2d", "f_per3d", "f_wall3d"])
def test_filter_matches_reference(name):
    f, sw, bc = G[f"{name}/f"], G[f"{name}/sw"], str(G[f"{name}/bc"])
    np.testing.assert_array_equal(ol.dccd_filter_nd(f, 0.05, bc), G[f"{name}/plain"])
    np.testing.assert_array_equal(ol.dccd_filter_nd(f, 0.05, bc, sw), G[f"{name}/switched"])


def test_filter_topology():
    """Periodic image kept; wall planes unfiltered (the reference's
    test_dccd_filter_preserves_periodic_image / _leaves_wall_boundaries_unfiltered)."""
    N = 32
    x = np.linspace(0.0, 1.0, N + 1)
    field = np.sin(2.0 * np.pi * x)[:, None] * np.ones((1, N + 1))
    out = ol.dccd_filter_nd(field, 0.05, "periodic_wall")
    assert np.max(np.abs(out[N, :] - out[0, :])) < 1e-14
    f = np.arange(17 * 17, dtype=float).reshape(17, 17)
    out = ol.dccd_filter_nd(f, 0.05, "wall")
    for sl in (np.s_[0, :], np.s_[-1, :], np.s_[:, 0], np.s_[:, -1]):
        np.testing.assert_array_equal(out[sl], f[sl])


@pytest.mark.parametrize("name", ["circle2d", "ellipse2d", "sphere3d"])
def test_curvature_matches_reference(name):
    N, L, bc, psi = G[f"{name}/N"], G[f"{name}/L"], str(G[f"{name}/bc"]), G[f"{name}/psi"]
    h = [float(L[a] / N[a]) for a in range(len(N))]
    for tag, kw in (("default", {}), ("nofilter", dict(dccd_eps=0.0)),
                    ("gauss", dict(gaussian_filter=True, psi_min=0.02))):
        key = f"{name}/kappa_{tag}"
        if key not in G:
            continue
        k = ol.curvature_psi(psi, h, bc, **kw)
        ref = G[key]
        scale = np.max(np.abs(ref))
        # the CCD line solves of the oracle and the reference differ in rounding
        np.testing.assert_allclose(k, ref, rtol=0, atol=1e-13 * scale)
        np.testing.assert_array_equal(k == 0.0, ref == 0.0)


def test_circle_curvature_value():
    """kappa ~ -1/R near a circle (reference test_curvature_psi_circle)."""
    N, R = 64, 0.25
    X, Y = np.meshgrid(np.linspace(0, 1, N + 1), np.linspace(0, 1, N + 1), indexing="ij")
    phi = np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2) - R
    eps = 1.5 / N
    psi = 1.0 / (1.0 + np.exp(-phi / eps))
    k = ol.curvature_psi(psi, [1.0 / N, 1.0 / N], "wall")
    near = np.abs(phi) < 2 * eps
    assert abs(np.mean(k[near]) + 1.0 / R) * R < 0.05


def test_properties_match_reference():
    rho, mu = ol.update_properties(G["props/psi"], 1.0, 0.001, 1.0, 0.0185)
    np.testing.assert_array_equal(rho, G["props/rho"])
    np.testing.assert_array_equal(mu, G["props/mu"])
