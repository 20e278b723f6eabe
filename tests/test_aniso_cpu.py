"""Anisotropic-kernel oracle against a direct transcription of the reference formulas.

The reference (Simulation/SurfaceReconstruction/AniKernelGenerator.cpp:53-101) computes,
for every particle p with neighbours q (|p - q| < r, q != p, r = kernelRatio x radius):

    W(d)    = 1 - (|d| / r)^3
    m       = (p + sum W(p - q) q) / (1 + sum W(p - q))       weighted mean
    centre  = lerp(p, m, positionBlending)
    C       = sum W(q - m) (q - m)(q - m)^T / (1 + sum W(q - m))     (>= threshold neighbours)
    U S V^T = svd(C);  S[i] = max(S[i], S[0] / axisRatio);  S *= cbrt(1 / prod S)
    kernel  = U diag(S) V^T          (spray points: defaultSpraySize x identity)

The transcription below uses brute-force neighbour lists, float64 sums and LAPACK's SVD;
the oracle (canonical order, float sums, Jacobi eigen-decomposition) must agree with it
to float rounding, and with the same spray classification.
"""
import numpy as np
import pytest

from oracle import oracle as O


def _reference_numpy(pos, radius, kernel_ratio=8.0, spray=0.75, blend=0.5, axis_ratio=8.0, threshold=25):
    pos = np.asarray(pos, np.float32)
    r = np.float32(kernel_ratio) * np.float32(radius)
    r2 = np.float32(r * r)
    n = len(pos)
    cen = np.zeros((n, 3))
    mat = np.zeros((n, 9))
    sprays = 0
    for p in range(n):
        d = pos[p] - pos                                    # float32, as the reference
        d2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        nb = np.nonzero(d2 < r2)[0]
        nb = nb[nb != p]
        q = pos[nb].astype(np.float64)
        w = 1.0 - (np.sqrt(d2[nb].astype(np.float64)) / float(r)) ** 3
        m = (pos[p].astype(np.float64) + (w[:, None] * q).sum(0)) / (1.0 + w.sum())
        cen[p] = (1.0 - blend) * pos[p] + blend * m
        if len(nb) < threshold:
            mat[p] = np.diag([spray] * 3).T.reshape(9)
            sprays += 1
            continue
        x = q - m
        dm = np.sqrt((x * x).sum(1))
        wm = np.where(dm < float(r), 1.0 - (dm / float(r)) ** 3, 0.0)
        C = (wm[:, None, None] * x[:, :, None] * x[:, None, :]).sum(0) / (1.0 + wm.sum())
        U, S, Vt = np.linalg.svd(C)
        S[1:] = np.maximum(S[1:], S[0] / axis_ratio)
        S *= np.cbrt(1.0 / np.prod(S))
        K = U @ np.diag(S) @ Vt
        mat[p] = K.T.reshape(9)                             # column-major (glm)
    return cen, mat, sprays


def _cloud(seed=5):
    """A dense block, a thin sheet and a few isolated spray points (cell size 1/32)."""
    rng = np.random.default_rng(seed)
    block = rng.uniform([0.1, 0.1, 0.1], [0.35, 0.3, 0.3], size=(1400, 3))
    sheet = np.stack([rng.uniform(0.5, 0.8, 500), rng.uniform(0.2, 0.5, 500), np.full(500, 0.6)], 1)
    sheet[:, 2] += rng.normal(0.0, 0.002, 500)
    spray = rng.uniform(0.05, 0.95, size=(40, 3))
    return np.concatenate([block, sheet, spray]).astype(np.float32)


def _grid_for(pos, cell):
    lo = pos.min(0).astype(np.float32)
    hi = pos.max(0).astype(np.float32)
    ext = ((hi - lo) / np.float32(cell)).astype(np.float32)
    return lo, np.floor(ext).astype(np.int32) + 1


@pytest.mark.parametrize("cell_factor", [0.25, 0.5, 1.0])
def test_oracle_matches_reference_formulas(cell_factor):
    pos = _cloud()
    radius = np.float32(1.0 / 64.0)            # kernel radius 8 x 1/64 = 0.125
    cell = np.float32(8.0 * radius * cell_factor)
    bmin, G = _grid_for(pos, cell)
    cen, mat, sprays = O.aniso_kernels(pos, bmin, cell, G, radius)
    rc, rm, rs = _reference_numpy(pos, radius)
    assert sprays == rs and 0 < sprays < len(pos)
    np.testing.assert_allclose(cen, rc, rtol=0, atol=2e-6)
    scale = np.abs(rm).max(1, keepdims=True)
    assert np.all(np.abs(mat - rm) <= 5e-5 * scale), np.abs(mat - rm).max()


def test_canonical_order_does_not_depend_on_grid_size_beyond_rounding():
    # different cell grids change only the summation order: float-rounding differences
    pos = _cloud(7)
    radius = np.float32(1.0 / 64.0)
    outs = []
    for f in (0.25, 1.0):
        cell = np.float32(8.0 * radius * f)
        bmin, G = _grid_for(pos, cell)
        outs.append(O.aniso_kernels(pos, bmin, cell, G, radius))
    assert outs[0][2] == outs[1][2]
    np.testing.assert_allclose(outs[0][0], outs[1][0], rtol=0, atol=1e-6)
    np.testing.assert_allclose(outs[0][1], outs[1][1], rtol=0, atol=1e-4)


def test_kernel_matrix_known_answers():
    # diag(4, 1, 1/4): the last axis is clamped to 4/8, then scaled to det 1 by cbrt(1/2)
    k = O.aniso_kernel_matrix(np.diag([4.0, 1.0, 0.25])).reshape(3, 3).T
    c = 0.5 ** (1.0 / 3.0)
    np.testing.assert_allclose(np.diag(k), [4 * c, c, 0.5 * c], rtol=1e-6)
    # an isotropic covariance gives the identity
    np.testing.assert_allclose(O.aniso_kernel_matrix(np.eye(3) * 3e-4).reshape(3, 3), np.eye(3), atol=1e-6)
    # a rotated SPD matrix: same eigen-structure, det 1, symmetric
    rng = np.random.default_rng(1)
    for _ in range(50):
        A = rng.normal(size=(3, 3))
        C = (A @ A.T) * 1e-3
        k = O.aniso_kernel_matrix(C).reshape(3, 3).T
        U, S, Vt = np.linalg.svd(C)
        S[1:] = np.maximum(S[1:], S[0] / 8.0)
        S *= np.cbrt(1.0 / np.prod(S))
        np.testing.assert_allclose(k, U @ np.diag(S) @ Vt, atol=2e-5 * np.abs(k).max())
        assert abs(np.linalg.det(k.astype(np.float64)) - 1.0) < 1e-4


def test_cbrt_newton():
    for v in [1.0, 8.0, 27.0, 0.125, 1e-30, 3.5e30, 2.0, 0.7]:
        assert abs(O.cbrt_newton(v) - np.cbrt(v)) <= 2 * np.spacing(np.cbrt(v))
    assert O.cbrt_newton(27.0) == 3.0 and O.cbrt_newton(-8.0) == -2.0
    assert O.cbrt_newton(0.0) == 0.0 and np.isinf(O.cbrt_newton(np.inf))


def test_line_of_points_elongates_the_kernel():
    # points on a line along x: the kernel's major axis is x, the others clamped to 1/8
    x = np.linspace(0.0, 1.0, 401, dtype=np.float32)
    pos = np.stack([x, np.full_like(x, 0.5), np.full_like(x, 0.5)], 1)
    pos[:, 1] += np.float32(1e-4) * np.sin(np.arange(401, dtype=np.float32))
    radius = np.float32(0.01)
    cell = np.float32(0.02)
    bmin, G = _grid_for(pos, cell)
    cen, mat, sprays = O.aniso_kernels(pos, bmin, cell, G, radius, threshold=10)
    k = mat[200].reshape(3, 3).T
    w, v = np.linalg.eigh(k)
    assert abs(abs(v[0, 2]) - 1.0) < 1e-3            # largest eigenvalue along x
    np.testing.assert_allclose(w[2] / w[:2], [8.0, 8.0], rtol=1e-3)
    # ends of the line have fewer neighbours than the middle but still > 10
    assert sprays == 0
