"""The device against the reference's own code, bit for bit.

The reference's RBFFD / TimeDependentPDE / CosineBell / VortexRollup,
compiled from its sources into oracle/_ref/libref_rbffd.so, compute every
multiply-add as a rounded product and a rounded sum (the reference's g++
-O3 build for x86-64 has no FMA).  With RBFFD_ARITH_UNFUSED the device's FP64
apply and stage kernels do the same, so on the reference's own weights
(uploaded with rbffd_weights_set) the device's derivatives and RK4 states
equal the reference's exactly.  The problems are the reference build's:
ONE_MONOMIAL (the constant is the only polynomial term), k-d tree stencils.
"""
import numpy as np
import pytest

import oracle as O
import rbffd_gpu_b200 as R

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.RefRBFFD.available(), reason="oracle/_ref/libref_rbffd.so not built")]

T_REV = 1036800.0


def _device_rbffd(ctx, ref, types):
    grid = R.Grid(ctx, ref.xyz, ref.stencils)
    der = R.RBFFD(types, grid, 2)
    for t in O.types_in_order(types):
        der.setWeights(t, np.ascontiguousarray(ref.weights(t)[:, :ref.n]))
    return grid, der


@pytest.fixture(scope="module")
def bell(ctx):
    N, n = 4096, 31  # the cosine bell at N = 4096, eps = 0.035 sqrt(N), LAMBDA + THETA + HV (k = 4)
    xyz = R.fibonacci_nodes(N, 1)
    ref = O.RefRBFFD(xyz, n, O.LAMBDA | O.THETA, 0.035 * np.sqrt(N), dim=2, hv_k=4, hv_gamma=1e-3, use_hv=True)
    grid, der = _device_rbffd(ctx, ref, R.LAMBDA | R.THETA | R.HV)
    yield ref, grid, der
    grid.close()
    ref.close()


def test_apply_unfused_equals_reference(ctx, bell):
    ref, grid, der = bell
    u = np.sin(3 * ref.xyz[:, 0]) + ref.xyz[:, 1] * ref.xyz[:, 2]
    ctx.setArithmetic(R.ARITH_UNFUSED)
    try:
        for t in (R.LAMBDA, R.THETA, R.HV):
            assert np.array_equal(der.applyWeightsForDeriv(t, u), ref.apply(t, u)), hex(t)
            got = der.applyWeightsForDeriv(t, u, start_indx=1000, nb_stencils=700)
            assert np.array_equal(got[1000:1700], ref.apply(t, u, 1000, 700)[1000:1700])
    finally:
        ctx.setArithmetic(R.ARITH_FUSED)
    # the default, fused arithmetic: within rounding of the reference, not equal to it
    d = der.applyWeightsForDeriv(R.LAMBDA, u)
    r = ref.apply(R.LAMBDA, u)
    assert np.abs(d - r).max() <= 1e-13 * np.abs(r).max()


@pytest.mark.parametrize("graph", [False, True])
def test_cosine_bell_unfused_equals_reference(bell, graph):
    ref, grid, der = bell
    h0 = R.exact_cosine_bell(ref.xyz)
    dt, steps = T_REV / 1000, 30
    want = ref.rk4(O.RefRBFFD.KIND_COSINE_BELL, h0, dt, steps, revolution=T_REV, use_hv=True)
    pde = R.CosineBell(grid, der, 1.0, np.pi / 2, T_REV, True, dtype=R.F64)
    pde.setArithmetic(R.ARITH_UNFUSED)
    assert pde.getArithmetic() == R.ARITH_UNFUSED and pde.getShape()[0] == 1
    pde.fillInitialConditions(h0)
    pde.advance(R.RK4, dt, steps, graph=graph)
    got = pde.getLocalSolution()
    pde.close()
    assert np.array_equal(got, want)


def test_cosine_bell_unfused_plain_path_equals_reference(bell):
    """The unfused path (one SpMV launch per operator, then the right-hand
    side and update) in the reference's arithmetic."""
    ref, grid, der = bell
    h0 = R.exact_cosine_bell(ref.xyz)
    dt = T_REV / 1000
    want = ref.rk4(O.RefRBFFD.KIND_COSINE_BELL, h0, dt, 5, revolution=T_REV, use_hv=True)
    pde = R.CosineBell(grid, der, 1.0, np.pi / 2, T_REV, True, dtype=R.F64)
    pde.setArithmetic(R.ARITH_UNFUSED)
    pde.fillInitialConditions(h0)
    pde.advance(R.RK4, dt, 5, unfused=True)
    got = pde.getLocalSolution()
    pde.close()
    assert np.array_equal(got, want)


def test_heat_unfused_equals_reference(ctx):
    N, n = 10242, 31
    xyz = R.fibonacci_nodes(N, 2)
    ref = O.RefRBFFD(xyz, n, O.LSFC, 0.25 / np.sqrt(4 * np.pi / N), dim=2)
    grid, der = _device_rbffd(ctx, ref, R.LSFC)
    try:
        u0 = R.exact_sph_heat(xyz, 8, np.random.default_rng(3).standard_normal(81), 0.0)
        want = ref.rk4(O.RefRBFFD.KIND_HEAT, u0, 1e-6, 40)
        ctx.setArithmetic(R.ARITH_UNFUSED)  # PDEs created now take the context's arithmetic
        try:
            pde = R.HeatSphere(grid, der, 1.0, dtype=R.F64)
        finally:
            ctx.setArithmetic(R.ARITH_FUSED)
        assert pde.getArithmetic() == R.ARITH_UNFUSED
        pde.fillInitialConditions(u0)
        pde.advance(R.RK4, 1e-6, 40, graph=True)
        assert np.array_equal(pde.getLocalSolution(), want)
        pde.close()
    finally:
        grid.close()
        ref.close()


def test_vortex_rollup_unfused_equals_reference(ctx):
    N, n = 4096, 31
    xyz = R.fibonacci_nodes(N, 4)
    ref = O.RefRBFFD(xyz, n, O.LAMBDA, 0.5 / np.sqrt(4 * np.pi / N), dim=2, hv_k=4, hv_gamma=1e-3, use_hv=True)
    grid, der = _device_rbffd(ctx, ref, R.LAMBDA | R.HV)
    try:
        h0 = R.exact_cosine_bell(xyz)
        want = ref.rk4(O.RefRBFFD.KIND_VORTEX, h0, 0.05, 20, use_hv=True)
        pde = R.VortexRollup(grid, der, True, dtype=R.F64)
        pde.setArithmetic(R.ARITH_UNFUSED)
        pde.fillInitialConditions(h0)
        pde.advance(R.RK4, 0.05, 20)
        assert np.array_equal(pde.getLocalSolution(), want)
        pde.close()
    finally:
        grid.close()
        ref.close()


def test_unfused_arithmetic_is_fp64_one_tracer_only(ctx, bell):
    ref, grid, der = bell
    p32 = R.CosineBell(grid, der, 1.0, np.pi / 2, T_REV, True, dtype=R.F32)
    with pytest.raises(R.RbffdError):
        p32.setArithmetic(R.ARITH_UNFUSED)
    p32.close()
    p64 = R.CosineBell(grid, der, 1.0, np.pi / 2, T_REV, True, dtype=R.F64)
    p64.setArithmetic(R.ARITH_UNFUSED)
    with pytest.raises(R.RbffdError):
        p64.setTiledShape(128, 1)
    with pytest.raises(R.RbffdError):
        p64.setShape(4, 256)
    p64.setArithmetic(R.ARITH_FUSED)  # back to the fused kernels and the autotuned shape
    assert p64.getArithmetic() == R.ARITH_FUSED
    p64.close()
