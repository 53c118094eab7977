"""Known answer of the reference's derivative driver
(tests/unified/evaluate_derivatives.cxx:301-512): X, Y, Z and LAPL weights on a
3-D node set applied to u = sin x + 2 cos y, compared with the analytic
derivatives cos x, -2 sin y, 0 and -sin x - 2 cos y through the reference's
norms (src/utils/norms.cpp), then the driver's mock RK4 chain
X u -> Y(X u) -> Z(Y X u) -> LAPL(Z Y X u) and its update
u_new = u + (X + 2 Y + 2 Z + L) / 6 (evaluate_derivatives.cxx:380-438).

The reference's grid files are not distributed; seeded uniform nodes in the
cube [-1, 1]^3 stand in, with interior nodes (|x|, |y|, |z| < 0.7) checked
separately since the one-sided stencils at the faces are less accurate.
"""
import numpy as np
import pytest

import oracle as O
import rbffd_gpu_b200 as R
from tests.helpers import rel_l2

N, n, EPS, DEG = 8000, 50, 1.0, 1
TYPES = O.X | O.Y | O.Z | O.LAPL


@pytest.fixture(scope="module")
def cube():
    rng = np.random.default_rng(11)
    xyz = rng.uniform(-1.0, 1.0, (N, 3))
    st = R.knn_stencils(xyz, n)
    x, y, z = xyz.T
    u = np.sin(x) + 2.0 * np.cos(y)
    exact = {O.X: np.cos(x), O.Y: -2.0 * np.sin(y), O.Z: np.zeros(N), O.LAPL: -np.sin(x) - 2.0 * np.cos(y)}
    inner = (np.abs(xyz) < 0.7).all(axis=1)
    return dict(xyz=xyz, st=st, u=u, exact=exact, inner=inner)


@pytest.fixture(scope="module")
def oracle_weights(cube):
    return O.weights(cube["xyz"], cube["st"], None, EPS, TYPES, dim=3, poly_deg=DEG)


def _check_against_analytic(derivs, cube):
    """rel. L2 (X, Y, LAPL) and absolute L-inf (Z, whose exact value is 0)."""
    ex, inner = cube["exact"], cube["inner"]
    for t, tol in ((O.X, 1e-4), (O.Y, 1e-4), (O.LAPL, 2e-3)):
        norms = R.sol_norms(derivs[t], ex[t])
        assert norms["l2_rel"] < tol, (t, norms)
        assert R.sol_norms(derivs[t][inner], ex[t][inner])["l2_rel"] < tol / 2, t
    assert np.abs(derivs[O.Z]).max() < 2e-3


def _mock_rk4(apply, u):
    dx = apply(O.X, u)
    dy = apply(O.Y, dx)
    dz = apply(O.Z, dy)
    dl = apply(O.LAPL, dz)
    return u + (1.0 / 6.0) * (dx + 2.0 * dy + 2.0 * dz + dl)


def test_oracle_derivatives_match_analytic(cube, oracle_weights):
    st, u = cube["st"], cube["u"]
    derivs = {t: O.apply(st, None, oracle_weights[t], u) for t in (O.X, O.Y, O.Z, O.LAPL)}
    _check_against_analytic(derivs, cube)


@pytest.mark.skipif(O.ref_lib("ref_norms") is None, reason="reference sources not built")
def test_driver_norms_are_the_reference_norms(cube, oracle_weights):
    """The product's norms equal the reference's norms.cpp (calcSolNorms' rule
    included) on the driver's error vectors, Z's all-zero exact value among them."""
    st, u = cube["st"], cube["u"]
    derivs = {t: O.apply(st, None, oracle_weights[t], u) for t in (O.X, O.Y, O.Z, O.LAPL)}
    for t in (O.X, O.Y, O.Z, O.LAPL):
        got = np.array([R.sol_norms(derivs[t], cube["exact"][t])[k] for k in ("l1", "l1_rel", "l2", "l2_rel", "linf", "linf_rel")])
        assert np.array_equal(got, O.ref_sol_norms(derivs[t], cube["exact"][t]))


@pytest.mark.gpu
def test_device_weights_and_apply_match_analytic_and_oracle(ctx, cube, oracle_weights):
    xyz, st, u = cube["xyz"], cube["st"], cube["u"]
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(TYPES, grid, 3)
    der.setEpsilon(EPS)
    der.setPolynomialDegree(DEG)
    der.computeAllWeightsForAllStencils()
    try:
        d64 = {t: der.applyWeightsForDeriv(t, u, dtype=R.F64) for t in (O.X, O.Y, O.Z, O.LAPL)}
        _check_against_analytic(d64, cube)
        for t in (O.X, O.Y, O.LAPL):
            do = O.apply(st, None, oracle_weights[t], u)
            assert rel_l2(d64[t], do) < 1e-6, t
            # FP64 apply of the device's own weights: bit for bit the oracle's SpMV
            assert np.array_equal(d64[t], O.apply(st, None, der.getWeights(t), u)), t
        d32 = {t: der.applyWeightsForDeriv(t, u, dtype=R.F32) for t in (O.X, O.Y, O.Z, O.LAPL)}
        _check_against_analytic(d32, cube)

        # the driver's chained applications and update, FP64 on the device against
        # the oracle's SpMV with the same weights
        W = {t: der.getWeights(t) for t in (O.X, O.Y, O.Z, O.LAPL)}
        got = _mock_rk4(lambda t, v: der.applyWeightsForDeriv(t, v, dtype=R.F64), u)
        ref = _mock_rk4(lambda t, v: O.apply(st, None, W[t], v), u)
        assert np.array_equal(got, ref)
    finally:
        grid.close()
