"""The CLS-transport oracle (FCCD flux-form right-hand side, TVD-RK3 step)
against the reference's own outputs (tests/golden/advect_golden.npz, written by
tests/golden/make_golden.py)."""

import os

import numpy as np
import pytest

from oracle import advect as oa

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "advect_golden.npz"))
CASES = ["wall2d", "per2d", "wall3d", "per3d"]


def _case(name):
    N, L, bc = G[f"{name}/N"], G[f"{name}/L"], str(G[f"{name}/bc"])
    vel = [G[f"{name}/u{a}"] for a in range(len(N))]
    return N, L, bc, vel, G[f"{name}/psi"], float(G[f"{name}/dt"])


@pytest.mark.parametrize("name", CASES)
def test_rhs_matches_reference(name):
    N, L, bc, vel, psi, dt = _case(name)
    np.testing.assert_array_equal(oa.flux_rhs(vel, psi, L, N, bc)[0], G[f"{name}/rhs_scalar"])
    mom = oa.flux_rhs(vel, None, L, N, bc)
    for a in range(len(N)):
        np.testing.assert_array_equal(mom[a], G[f"{name}/rhs_mom{a}"])


@pytest.mark.parametrize("name", CASES)
def test_rk3_step_matches_reference(name):
    N, L, bc, vel, psi, dt = _case(name)
    np.testing.assert_array_equal(oa.advance(psi, vel, dt, L, N, bc), G[f"{name}/psi_new"])
    np.testing.assert_array_equal(oa.advance(psi, vel, dt, L, N, bc, clip=None), G[f"{name}/psi_new_noclip"])


@pytest.mark.parametrize("name", CASES)
def test_node_mode_matches_reference(name):
    """Option C: node gradients, the nodal right-hand sides and one RK3 step in
    node mode, bit for bit."""
    N, L, bc, vel, psi, dt = _case(name)
    from oracle import ccd as occd
    from oracle.levelset import axis_kinds
    kinds = axis_kinds(bc, len(N))
    for a in range(len(N)):
        H = float(np.linspace(0.0, L[a], N[a] + 1)[1])
        q = occd.differentiate(psi, a, float(L[a] / N[a]), bc=kinds[a])[1]
        np.testing.assert_array_equal(oa.node_gradient(psi, q, a, H, kinds[a] == "periodic"),
                                      G[f"{name}/node_grad_psi{a}"])
    np.testing.assert_array_equal(oa.node_rhs(vel, psi, L, N, bc)[0], G[f"{name}/rhs_scalar_node"])
    mom = oa.node_rhs(vel, None, L, N, bc)
    for a in range(len(N)):
        np.testing.assert_array_equal(mom[a], G[f"{name}/rhs_mom_node{a}"])
    np.testing.assert_array_equal(oa.advance(psi, vel, dt, L, N, bc, mode="node"), G[f"{name}/psi_new_node"])


def test_flux_form_conserves_on_a_periodic_box():
    """sum over the unique nodes of -div(F) vanishes (telescoping faces)."""
    rng = np.random.default_rng(3)
    N, L = (12, 10), (1.0, 1.0)
    vel = [rng.standard_normal((13, 11)) for _ in range(2)]
    psi = rng.uniform(0.0, 1.0, (13, 11))
    for v in vel + [psi]:
        oa.sync_images(v, "periodic")
    r = oa.flux_rhs(vel, psi, L, N, "periodic")[0]
    assert abs(r[:-1, :-1].sum()) < 1e-10 * np.abs(r).sum()


R = np.load(os.path.join(os.path.dirname(__file__), "golden", "reinit_golden.npz"))
REINIT = ["zero2d", "per2d", "neu2d", "zero3d"]


def reinit_args(g, name):
    N = tuple(int(x) for x in g[f"{name}/N"])
    L = tuple(float(x) for x in g[f"{name}/L"])
    return (L, N, str(g[f"{name}/ccd_bc"]), float(g[f"{name}/eps"]), int(g[f"{name}/n_steps"]), str(g[f"{name}/bc"]),
            0.05, bool(g[f"{name}/mass"]))


@pytest.mark.parametrize("name", REINIT)
def test_reinit_matches_reference(name):
    """Split reinitialization (zero / periodic / neumann ghost padding, with and
    without mass correction) equals the reference bit for bit."""
    np.testing.assert_array_equal(oa.reinitialize(R[f"{name}/psi"], *reinit_args(R, name)), R[f"{name}/psi_reinit"])


@pytest.mark.parametrize("name", CASES)
def test_mass_corrected_transport_matches_reference(name):
    N, L, bc, vel, psi, dt = _case(name)
    q = oa.advance(psi, vel, dt, L, N, bc)
    dV = oa.cell_volumes(L, N, oa.periodic_flags(bc, len(N)))
    target = np.sum(oa.sync_images(psi.copy(), bc) * dV)
    np.testing.assert_array_equal(oa.sync_images(oa.mass_correction(q, dV, target), bc), G[f"{name}/psi_new_mass"])


@pytest.mark.parametrize("name", CASES)
def test_uccd6_matches_reference(name):
    """UCCD6 skew convection + hyperviscosity (five CCD solves per pair)."""
    N, L, bc, vel, psi, dt = _case(name)
    u = oa.uccd6(vel, L, N, bc)
    for a in range(len(N)):
        np.testing.assert_array_equal(u[a], G[f"{name}/uccd6_{a}"])
