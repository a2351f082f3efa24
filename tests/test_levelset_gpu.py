"""GPU tests of curvature from psi, the DCCD filter and the material
properties, against the reference's outputs (tests/golden/levelset_golden.npz)
and the oracle."""

from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import levelset as ol

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "levelset_golden.npz")
# the CCD derivatives agree with the reference to ~1e-13 relative (test_ccd_gpu);
# kappa divides by |grad psi|^3, which costs a few more digits near the mask edge
TOL = 1e-10
KW = {"default": {}, "nofilter": dict(dccd_eps=0.0), "gauss": dict(gaussian_filter=True, psi_min=0.02)}


@pytest.fixture(scope="module")
def golden():
    with np.load(GOLDEN) as d:
        return {k: d[k] for k in d.files}


def _ccd(N, L, bc, dtype=None):
    from twophaseflow_b200 import CCDSolver, UniformGrid
    return CCDSolver(UniformGrid(tuple(N), tuple(L)), None, bc_type=bc, dtype=dtype)


@pytest.mark.parametrize("name", ["circle2d", "ellipse2d", "sphere3d"])
def test_curvature_matches_reference(cuda_device, golden, name):
    from twophaseflow_b200 import CurvatureCalculatorPsi
    N = [int(n) for n in golden[f"{name}/N"]]
    L = [float(x) for x in golden[f"{name}/L"]]
    ccd = _ccd(N, L, str(golden[f"{name}/bc"]))
    psi = golden[f"{name}/psi"]
    for tag, kw in KW.items():
        key = f"{name}/kappa_{tag}"
        if key not in golden:
            continue
        k = CurvatureCalculatorPsi(None, ccd, **kw).compute(psi)
        ref = golden[key]
        assert isinstance(k, np.ndarray) and k.shape == ref.shape
        assert np.abs(k - ref).max() <= TOL * np.abs(ref).max(), (key, np.abs(k - ref).max())
        if tag != "gauss":
            assert np.array_equal(k == 0.0, ref == 0.0)


@pytest.mark.parametrize("name", ["f_wall2d", "f_pw2d", "f_per3d", "f_wall3d"])
def test_filter_bit_exact(cuda_device, golden, name):
    """Same operations in the same order as the reference: bit-identical."""
    from twophaseflow_b200 import dccd_filter_nd
    f, sw, bc = golden[f"{name}/f"], golden[f"{name}/sw"], str(golden[f"{name}/bc"])
    np.testing.assert_array_equal(dccd_filter_nd(f, None, 0.05, bc_type=bc), golden[f"{name}/plain"])
    np.testing.assert_array_equal(dccd_filter_nd(f, None, 0.05, bc_type=bc, switch=sw), golden[f"{name}/switched"])


@pytest.mark.parametrize("bc", ["wall", "periodic"])
def test_filter_full_size_against_oracle(cuda_device, bc):
    """257^3 nodes (136 MB per field, larger than L2): bit-exact against the oracle."""
    import torch
    from twophaseflow_b200 import dccd_filter_nd
    rng = np.random.default_rng(5)
    f = rng.standard_normal((257, 257, 257))
    sw = rng.uniform(0.0, 1.0, f.shape)
    ft = torch.from_numpy(f).cuda()
    st = torch.from_numpy(sw).cuda()
    out = dccd_filter_nd(ft, None, 0.05, bc_type=bc, switch=st)
    assert out.is_cuda
    np.testing.assert_array_equal(out.cpu().numpy(), ol.dccd_filter_nd(f, 0.05, bc, sw))


def test_curvature_3d_against_oracle(cuda_device):
    """65^3 sphere on a wall box against the oracle; device tensors in and out."""
    import torch
    from twophaseflow_b200 import CurvatureCalculatorPsi
    N, L = (64, 64, 64), (1.0, 1.0, 1.0)
    X = np.meshgrid(*[np.linspace(0.0, 1.0, n + 1) for n in N], indexing="ij")
    phi = np.sqrt((X[0] - 0.5) ** 2 + (X[1] - 0.48) ** 2 + (X[2] - 0.52) ** 2) - 0.3
    eps = 1.5 / 64
    psi = 1.0 / (1.0 + np.exp(-phi / eps))
    k = CurvatureCalculatorPsi(None, _ccd(N, L, "wall")).compute(torch.from_numpy(psi).cuda())
    assert k.is_cuda
    ref = ol.curvature_psi(psi, [1.0 / 64] * 3, "wall")
    k = k.cpu().numpy()
    assert np.abs(k - ref).max() <= TOL * np.abs(ref).max()
    # kappa of a sphere: the sum of both principal curvatures, -2/R
    near = np.abs(phi) < eps
    assert abs(np.mean(k[near]) * 0.3 / 2.0 + 1.0) < 0.05


def test_curvature_circle_large_f32(cuda_device):
    """1025^2 circle (size-independent check): -1/R near the interface in FP64
    and FP32, FP32 within 1e-3 of FP64 there."""
    import torch
    from twophaseflow_b200 import CurvatureCalculatorPsi
    N, R = 1024, 0.25
    x = np.linspace(0.0, 1.0, N + 1)
    X, Y = np.meshgrid(x, x, indexing="ij")
    phi = np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2) - R
    eps = 1.5 / N
    psi = 1.0 / (1.0 + np.exp(-phi / eps))
    near = np.abs(phi) < 2 * eps
    k64 = CurvatureCalculatorPsi(None, _ccd((N, N), (1.0, 1.0), "wall")).compute(psi)
    assert abs(np.mean(k64[near]) * R + 1.0) < 0.01
    k32 = CurvatureCalculatorPsi(None, _ccd((N, N), (1.0, 1.0), "wall", torch.float32)).compute(psi)
    assert k32.dtype == np.float32
    assert np.abs(k32[near] - k64[near]).max() <= 1e-3 * np.abs(k64[near]).max()


def test_properties_bit_exact(cuda_device, golden):
    from twophaseflow_b200 import update_properties
    rho, mu = update_properties(None, golden["props/psi"], 1.0, 0.001, 1.0, 0.0185)
    np.testing.assert_array_equal(rho, golden["props/rho"])
    np.testing.assert_array_equal(mu, golden["props/mu"])


def test_filter_refuses_aliasing(cuda_device):
    import ctypes as C
    import torch
    from twophaseflow_b200 import _lib
    f = torch.zeros((8, 8), dtype=torch.float64, device="cuda")
    t = torch.empty_like(f)
    shape = (C.c_int64 * 2)(8, 8)
    per = (C.c_int * 2)(0, 0)
    st = _lib.load().tpf_dccd_filter(2, shape, per, 0.05, None, _lib.dptr(f), _lib.dptr(f), _lib.dptr(t),
                                     _lib.TPF_F64, None)
    assert st != 0 and "distinct" in _lib.last_error()
