"""Edge cases of the device path: grids smaller than one halo tile, stencils
of the centre alone, empty subranges, zero steps, systems past the solver's
size limit and non-finite states."""
import numpy as np
import pytest

import oracle as O
import rbffd_gpu_b200 as R
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


def test_tiny_grid_end_to_end(ctx):
    """40 nodes, 10-node stencils (fewer rows than one 64-row tile): device
    weights, apply and heat RK4 against the oracle; one lane per row equals
    the oracle bit for bit on the device's own weights."""
    N, n = 40, 10
    xyz = R.fibonacci_nodes(N, 11)
    st = R.knn_stencils(xyz, n)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(R.LSFC, grid, 2)
    der.setEpsilon(2.0)
    der.setPolynomialDegree(1)
    der.computeAllWeightsForAllStencils()
    W = der.getWeights(R.LSFC)
    Wo = O.weights(xyz, st, None, 2.0, O.LSFC, dim=2, poly_deg=1)[O.LSFC]
    assert np.isfinite(W).all()
    f = np.sin(xyz[:, 0]) + xyz[:, 2]
    assert rel_l2(O.apply(st, None, W, f), O.apply(st, None, Wo, f)) < 1e-8
    assert np.array_equal(der.applyWeightsForDeriv(R.LSFC, f), O.apply(st, None, W, f))
    u0 = np.cos(2 * xyz[:, 1])
    for shape in ((1, 256), None):
        pde = R.HeatSphere(grid, der, 1.0, dtype=R.F64)
        if shape:
            pde.setShape(*shape)
        pde.fillInitialConditions(u0)
        pde.advance(R.RK4, 1e-3, 7, graph=True)
        out = pde.getLocalSolution()
        pde.close()
        ref = O.rk4_heat(st, None, W, u0, 1e-3, 7)
        if shape:
            assert np.array_equal(out, ref)
        else:
            assert rel_l2(out, ref) <= 1e-13
    grid.close()


def test_single_node_stencils(ctx):
    """Stencils of the centre alone with the constant polynomial: the
    2 x 2 system [phi(0) 1; 1 0] gives weight 0 for a derivative (it must
    annihilate constants), so the derivative of anything is 0."""
    N = 256
    xyz = R.fibonacci_nodes(N, 12)
    st = np.arange(N, dtype=np.int32)[:, None]
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(R.LSFC | R.XSFC, grid, 2)
    der.setEpsilon(3.0)
    der.setPolynomialDegree(0)
    der.computeAllWeightsForAllStencils()
    for t in (R.LSFC, R.XSFC):
        w = der.getWeights(t)
        assert np.all(w == 0.0)
        assert np.all(der.applyWeightsForDeriv(t, np.random.default_rng(1).random(N)) == 0.0)
    grid.close()


def test_empty_subrange_and_zero_steps(ctx):
    """An apply over no stencils leaves the output untouched; advancing by
    zero steps leaves the state and the time unchanged."""
    N, n = 512, 13
    xyz = R.fibonacci_nodes(N, 13)
    st = R.knn_stencils(xyz, n)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(R.LSFC, grid, 2)
    der.setEpsilon(4.0)
    der.setPolynomialDegree(1)
    der.computeAllWeightsForAllStencils()
    out = np.full(N, 7.0)
    der.applyWeightsForDeriv(R.LSFC, np.ones(N), deriv=out, start_indx=100, nb_stencils=0)
    assert np.all(out == 7.0)
    pde = R.HeatSphere(grid, der, 1.0, dtype=R.F64)
    u0 = np.random.default_rng(2).random(N)
    pde.fillInitialConditions(u0)
    pde.advance(R.RK4, 1e-3, 0)
    assert np.array_equal(pde.getLocalSolution(), u0)
    assert pde.getTime() == 0.0
    pde.close()
    grid.close()


def test_system_past_the_size_limit_is_refused(ctx):
    """150-node stencils with degree-4 polynomials make 165 unknowns, past the
    solver's 160: the call reports it and computes nothing."""
    N, n = 2000, 150
    xyz = R.fibonacci_nodes(N, 14)
    st = R.knn_stencils(xyz, n)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(R.XSFC, grid, 2)
    der.setEpsilon(10.0)
    der.setPolynomialDegree(4)
    with pytest.raises(R.RbffdError) as e:
        der.computeAllWeightsForAllStencils()
    assert e.value.status == -5  # RBFFD_ERR_UNSUPPORTED
    der.setPolynomialDegree(2)  # 156 unknowns: within the limit
    der.computeAllWeightsForAllStencils()
    assert np.isfinite(der.getWeights(R.XSFC)).all()
    grid.close()


def test_non_finite_state_stays_local(ctx):
    """A NaN in the state spreads only through the stencils that read it:
    after one RK4 step the rows whose stencils avoid the node stay finite."""
    N, n = 4096, 13
    xyz = R.fibonacci_nodes(N, 15)
    st = R.knn_stencils(xyz, n)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(R.LSFC, grid, 2)
    der.setEpsilon(8.0)
    der.setPolynomialDegree(1)
    der.computeAllWeightsForAllStencils()
    u0 = np.ones(N)
    u0[123] = np.nan
    pde = R.HeatSphere(grid, der, 1.0, dtype=R.F64)
    pde.fillInitialConditions(u0)
    pde.advance(R.RK4, 1e-6, 1)
    out = pde.getLocalSolution()
    pde.close()
    # each of the 4 stages applies the operator once: the NaN reaches at most 4 stencil hops
    reach = np.zeros(N, dtype=bool)
    reach[123] = True
    for _ in range(4):
        reach |= np.isin(st, np.flatnonzero(reach)).any(axis=1)
    assert np.isnan(out[123])
    assert np.isfinite(out[~reach]).all()
    assert (~reach).sum() > N // 2
    grid.close()
