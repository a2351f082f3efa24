"""The viscous-stress oracle against the reference's own outputs
(tests/golden/viscous_golden.npz, written by tests/golden/make_golden.py)."""

import os

import numpy as np
import pytest

from oracle import viscous as ov

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "viscous_golden.npz"))
SCHEMES = ["ccd_bulk", "conservative_stress", "ccd_stress_legacy"]


@pytest.mark.parametrize("name", ["wall2d", "per2d", "wall3d"])
@pytest.mark.parametrize("scheme", SCHEMES)
def test_viscous_matches_reference(name, scheme):
    N, L, bc = G[f"{name}/N"], G[f"{name}/L"], str(G[f"{name}/bc"])
    vel = [G[f"{name}/u{a}"] for a in range(len(N))]
    v = ov.viscous(vel, G[f"{name}/mu"], G[f"{name}/rho"], 100.0, L, N, bc, scheme)
    for a in range(len(N)):
        np.testing.assert_array_equal(v[a], G[f"{name}/{scheme}/v{a}"])


def test_low_order_derivative_exact_on_quadratics():
    """The three-point stencil differentiates x^2 exactly on a uniform grid."""
    x = np.linspace(0.0, 1.0, 33)
    d = ov.low_order_derivative(x ** 2, 0, x)
    assert np.abs(d[1:-1] - 2.0 * x[1:-1]).max() < 1e-12


@pytest.mark.parametrize("name", ["wall2d", "per2d", "wall3d"])
@pytest.mark.parametrize("tag,cn", [("cn", True), ("fe", False)])
def test_cn_predictor_matches_reference(name, tag, cn):
    """ViscousTerm.apply_cn_predictor: Picard CN (Heun) and forward Euler."""
    N, L, bc = G[f"{name}/N"], G[f"{name}/L"], str(G[f"{name}/bc"])
    vel = [G[f"{name}/u{a}"] for a in range(len(N))]
    e = [G[f"{name}/e{a}"] for a in range(len(N))]
    u = ov.cn_predictor(vel, e, G[f"{name}/mu"], G[f"{name}/rho"], 100.0, L, N, bc, 0.003, cn)
    for a in range(len(N)):
        np.testing.assert_array_equal(u[a], G[f"{name}/pred_{tag}{a}"])


@pytest.mark.parametrize("name", ["wall2d", "per2d", "wall3d"])
def test_interface_band_ccd_bulk_matches_reference(name):
    """ccd_bulk with psi given (interface band: normal-axis low-order /
    tangential CCD stress divergence; bulk: mu times the CCD Laplacian),
    bit for bit; both branches occur in every case."""
    N, L, bc = G[f"{name}/N"], G[f"{name}/L"], str(G[f"{name}/bc"])
    vel = [G[f"{name}/u{a}"] for a in range(len(N))]
    psi = G[f"{name}/psi"]
    coords = [np.linspace(0.0, L[a], N[a] + 1) for a in range(len(N))]
    band, _ = ov.band_masks(psi, coords)
    assert band.any() and (~band).any()
    v = ov.viscous(vel, G[f"{name}/mu"], G[f"{name}/rho"], 100.0, L, N, bc, "ccd_bulk", psi=psi)
    for a in range(len(N)):
        np.testing.assert_array_equal(v[a], G[f"{name}/ccd_bulk_band/v{a}"])


@pytest.mark.parametrize("name", ["wall2d", "per2d", "wall3d"])
def test_cn_predictor_richardson_matches_reference(name):
    """cn_mode='richardson_picard': the reference's RichardsonCNAdvance around
    Picard, bit for bit."""
    N, L, bc = G[f"{name}/N"], G[f"{name}/L"], str(G[f"{name}/bc"])
    vel = [G[f"{name}/u{a}"] for a in range(len(N))]
    e = [G[f"{name}/e{a}"] for a in range(len(N))]
    u = ov.cn_predictor_richardson(vel, e, G[f"{name}/mu"], G[f"{name}/rho"], 100.0, L, N, bc, 0.003)
    for a in range(len(N)):
        np.testing.assert_array_equal(u[a], G[f"{name}/pred_rich{a}"])


P = np.load(os.path.join(os.path.dirname(__file__), "golden", "predictor_golden.npz"))


def predictor_states(g, name):
    nd = len(g[f"{name}/N"])
    states, dts = [], []
    for s in range(2):
        vel = [g[f"{name}/s{s}/u{a}"] for a in range(nd)]
        psi = g[f"{name}/s{s}/psi"]
        states.append((vel, 0.1 + 0.9 * psi, 0.01 + 0.99 * psi, g[f"{name}/s{s}/kappa"], psi, g[f"{name}/s{s}/p"]))
        dts.append(float(g[f"{name}/s{s}/dt"]))
    return states, dts


@pytest.mark.parametrize("name", ["wall2d", "per2d", "wall3d"])
def test_predictor_matches_reference(name):
    """Two Predictor.compute calls (forward Euler then AB2 convection; CN or
    explicit viscous; CSF or GFM) equal the reference bit for bit."""
    N = tuple(int(x) for x in P[f"{name}/N"])
    L = tuple(float(x) for x in P[f"{name}/L"])
    states, dts = predictor_states(P, name)
    outs = ov.predictor_steps(states, dts, 50.0, 0.8, 4.0, L, N, str(P[f"{name}/bc"]), bool(P[f"{name}/cn"]),
                              bool(P[f"{name}/gfm"]))
    for s in range(2):
        for a in range(len(N)):
            np.testing.assert_array_equal(outs[s][a], P[f"{name}/s{s}/ustar{a}"])
