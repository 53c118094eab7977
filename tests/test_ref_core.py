"""The oracle against the reference's own hot path, compiled from its sources
(oracle/ref_rbffd.cpp -> oracle/_ref/libref_rbffd.so): RBFFD's weights,
getStencilLHS / getStencilMultiRHS, both applyWeightsForDeriv overloads,
TimeDependentPDE::advanceRungeKutta4 with CosineBell, VortexRollup and the
sphere heat right-hand side, and the cosine-bell experiment's ExactAdvection.

The reference build computes with a rounded product and a rounded sum for
every multiply-add (its g++ -O3 flags for x86-64 have no FMA), so the
oracle runs in that arithmetic here (oracle.reference_arithmetic); its
default, fused model is the device's FP64 arithmetic, and the last test
bounds the distance between the two.  Every comparison but that one is bit
for bit.  The reference build has ONE_MONOMIAL set (rbffd.cpp:1), so the
oracle runs with polynomial degree 0 (the constant) against it.
"""
import numpy as np
import pytest

import oracle as O
import rbffd_gpu_b200 as R

pytestmark = pytest.mark.skipif(not O.RefRBFFD.available(),
                                reason="oracle/_ref/libref_rbffd.so not built (needs the reference tree)")

T_REV = 1036800.0  # one revolution in 1000 steps of 1036.8 s (cosine-bell experiment, test.conf)


def _hv_scale(gamma, k, N):
    # RBFFD::getHVScalar (rbffd.h:227-238): -hv_gamma * N^-hv_k
    return -gamma * float(N) ** (-float(k))


@pytest.fixture(scope="module")
def bell():
    """The C1 cosine bell at the reference's own basis: N = 4096 Fibonacci
    nodes, n = 31, eps = 0.035 sqrt(N), LAMBDA + THETA + HV (k = 4, dim 2,
    gamma = 1e-3)."""
    N, n = 4096, 31
    xyz = R.fibonacci_nodes(N, 1)
    eps = 0.035 * np.sqrt(N)
    ref = O.RefRBFFD(xyz, n, O.LAMBDA | O.THETA, eps, dim=2, hv_k=4, hv_gamma=1e-3, use_hv=True)
    yield xyz, ref, eps
    ref.close()


def test_reference_stencils_are_the_product_stencils(bell):
    xyz, ref, _ = bell
    assert np.array_equal(ref.stencils, R.knn_stencils(xyz, ref.n))


def test_weights_equal_reference_cosine_bell(bell):
    xyz, ref, eps = bell
    N, n = ref.N, ref.n
    W = O.weights(xyz, ref.stencils, None, eps, O.LAMBDA | O.THETA | O.HV, dim=2, poly_deg=0, hv_k=4,
                  hv_scale=_hv_scale(1e-3, 4, N))
    for t in (O.LAMBDA, O.THETA, O.HV):
        assert np.array_equal(ref.weights(t)[:, :n], W[t]), hex(t)


@pytest.mark.parametrize("types,dim", [
    (O.LSFC, 2),
    (O.X | O.Y | O.Z | O.LAPL, 3),
    (O.XSFC | O.YSFC | O.ZSFC, 2),
    (O.R | O.INTERP | O.LAPL, 2),
])
def test_weights_equal_reference_other_operators(types, dim):
    N, n = 1200, 17
    xyz = R.fibonacci_nodes(N, 5)
    eps = 0.3 / np.sqrt(4 * np.pi / N)
    ref = O.RefRBFFD(xyz, n, types, eps, dim=dim)
    try:
        W = O.weights(xyz, ref.stencils, None, eps, types, dim=dim, poly_deg=0)
        for t in O.types_in_order(types):
            assert np.array_equal(ref.weights(t)[:, :n], W[t]), hex(t)
    finally:
        ref.close()


def test_alt_sfc_weights_equal_reference():
    """ALT_XSFC/YSFC/ZSFC: the reference computes X, Y, Z and projects them
    (rbffd.cpp:337-347)."""
    N, n = 1200, 17
    xyz = R.fibonacci_nodes(N, 6)
    eps = 0.3 / np.sqrt(4 * np.pi / N)
    ALT = 0x1000 | 0x2000 | 0x4000
    ref = O.RefRBFFD(xyz, n, ALT, eps, dim=3)
    try:
        W = O.weights(xyz, ref.stencils, None, eps, O.X | O.Y | O.Z, dim=3, poly_deg=0)
        ax, ay, az = O.alt_sfc(xyz, W[O.X], W[O.Y], W[O.Z])
        for t, a in ((0x1000, ax), (0x2000, ay), (0x4000, az)):
            assert np.array_equal(ref.weights(t)[:, :n], a), hex(t)
    finally:
        ref.close()


def test_stencil_systems_equal_reference(bell):
    """getStencilLHS (with distanceMatrix) and getStencilMultiRHS, one column
    per selected DerType in bit order, against the oracle's assembly."""
    xyz, ref, eps = bell
    for i in (0, 17, 1000, 4095):
        A, B = ref.system(i, 3)
        aug = O.assemble(xyz, ref.stencils[i], 0, eps, O.LAMBDA | O.THETA | O.HV, dim=2, hv_k=4)
        m = ref.n + 1
        assert np.array_equal(A, aug[:, :m]), i
        assert np.array_equal(B, aug[:, m:]), i


def test_apply_equals_reference_both_overloads(bell):
    xyz, ref, _ = bell
    n = ref.n
    u = np.sin(3 * xyz[:, 0]) + xyz[:, 1] * xyz[:, 2]
    with O.reference_arithmetic():
        for t in (O.LAMBDA, O.THETA, O.HV):
            w = np.ascontiguousarray(ref.weights(t)[:, :n])
            assert np.array_equal(ref.apply(t, u), O.apply(ref.stencils, None, w, u)), hex(t)
            # the pointer overload over a sub-range (rows outside it untouched: 0)
            sub = ref.apply(t, u, 1000, 700)
            full = O.apply(ref.stencils, None, w, u)
            assert np.array_equal(sub[1000:1700], full[1000:1700])
            assert not sub[:1000].any() and not sub[1700:].any()


def test_rk4_cosine_bell_equals_reference(bell):
    """CosineBell::solve + TimeDependentPDE::advanceRungeKutta4, 10 steps of
    the experiment's dt from the bell's initial state."""
    xyz, ref, _ = bell
    n = ref.n
    h0 = R.exact_cosine_bell(xyz)
    dt = T_REV / 1000
    got = ref.rk4(O.RefRBFFD.KIND_COSINE_BELL, h0, dt, 10, revolution=T_REV, use_hv=True)
    W = {t: np.ascontiguousarray(ref.weights(t)[:, :n]) for t in (O.LAMBDA, O.THETA, O.HV)}
    cu, cv = O.cosine_bell_coeffs(xyz, 1.0, np.pi / 2, 2 * np.pi / T_REV)
    with O.reference_arithmetic():
        want = O.rk4_advect(ref.stencils, None, W[O.LAMBDA], W[O.THETA], W[O.HV], cu, cv, h0, dt, 10)
    assert np.array_equal(got, want)
    # without hyperviscosity in the right-hand side
    got = ref.rk4(O.RefRBFFD.KIND_COSINE_BELL, h0, dt, 3, revolution=T_REV, use_hv=False)
    with O.reference_arithmetic():
        want = O.rk4_advect(ref.stencils, None, W[O.LAMBDA], W[O.THETA], None, cu, cv, h0, dt, 3)
    assert np.array_equal(got, want)


def test_rk4_heat_equals_reference():
    """The sphere heat equation (right-hand side W_LSFC u through the
    reference's applyWeightsForDeriv) under advanceRungeKutta4."""
    N, n = 2562, 31
    xyz = R.fibonacci_nodes(N, 2)
    eps = 0.25 / np.sqrt(4 * np.pi / N)
    ref = O.RefRBFFD(xyz, n, O.LSFC, eps, dim=2)
    try:
        u0 = R.exact_sph_heat(xyz, 8, np.random.default_rng(3).standard_normal(81), 0.0)
        got = ref.rk4(O.RefRBFFD.KIND_HEAT, u0, 1e-5, 12)
        W = np.ascontiguousarray(ref.weights(O.LSFC)[:, :n])
        with O.reference_arithmetic():
            want = O.rk4_heat(ref.stencils, None, W, u0, 1e-5, 12)
        assert np.array_equal(got, want)
    finally:
        ref.close()


def test_rk4_vortex_rollup_equals_reference():
    """VortexRollup::solve (f = -w(theta) D_lambda h + H h) under advanceRungeKutta4."""
    N, n = 2562, 31
    xyz = R.fibonacci_nodes(N, 4)
    eps = 0.5 / np.sqrt(4 * np.pi / N)
    ref = O.RefRBFFD(xyz, n, O.LAMBDA, eps, dim=2, hv_k=4, hv_gamma=1e-3, use_hv=True)
    try:
        h0 = R.exact_cosine_bell(xyz)
        got = ref.rk4(O.RefRBFFD.KIND_VORTEX, h0, 0.05, 8, use_hv=True)
        wl = np.ascontiguousarray(ref.weights(O.LAMBDA)[:, :n])
        wh = np.ascontiguousarray(ref.weights(O.HV)[:, :n])
        w = O.vortex_rollup_w(xyz)
        with O.reference_arithmetic():
            want = O.rk4_advect(ref.stencils, None, wl, np.zeros_like(wl), wh, w, np.zeros(N), h0, 0.05, 8)
        assert np.array_equal(got, want)
    finally:
        ref.close()


def test_exact_cosine_bell_equals_reference_exact_advection():
    """rbffd_exact_cosine_bell against the experiment's ExactAdvection
    (exact_advection.h:37-53), compiled from the reference."""
    for N, seed in ((4096, 1), (10242, 9)):
        xyz = R.fibonacci_nodes(N, seed)
        for a in (1.0, 6.37122e6):
            assert np.array_equal(R.exact_cosine_bell(xyz * a, a), O.ref_exact_advection(xyz * a, a, 0.0))


def test_fused_model_within_rounding_of_the_reference(bell):
    """The device's arithmetic (one rounding per multiply-add) against the
    reference's (two): after 10 cosine-bell steps the two agree to a few
    units in the last place of the solution's scale."""
    xyz, ref, _ = bell
    n = ref.n
    h0 = R.exact_cosine_bell(xyz)
    dt = T_REV / 1000
    got = ref.rk4(O.RefRBFFD.KIND_COSINE_BELL, h0, dt, 10, revolution=T_REV, use_hv=True)
    W = {t: np.ascontiguousarray(ref.weights(t)[:, :n]) for t in (O.LAMBDA, O.THETA, O.HV)}
    cu, cv = O.cosine_bell_coeffs(xyz, 1.0, np.pi / 2, 2 * np.pi / T_REV)
    fused = O.rk4_advect(ref.stencils, None, W[O.LAMBDA], W[O.THETA], W[O.HV], cu, cv, h0, dt, 10)
    assert not np.array_equal(fused, got)  # the two models do differ ...
    assert np.abs(fused - got).max() <= 1e-13 * np.abs(got).max()  # ... by rounding only
