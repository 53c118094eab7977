"""Cluster-resident RK4 (RBFFD_ADVANCE_RESIDENT): every step in one launch of
a thread-block cluster (up to 16 CTAs) holding the weights (in registers for
31- and 50-node stencils), stencils, halos and state on chip.  It performs the one-lane-per-row kernels'
arithmetic, so it must give their bits (and, in FP64, the oracle's)."""
import numpy as np
import pytest

import oracle as O
import rbffd_gpu_b200 as R
from tests.helpers import sphere_problem, cosine_bell_setup

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bell(ctx):
    N, n = 4096, 31
    xyz, st = sphere_problem(N, n, 1)
    types = O.LAMBDA | O.THETA | O.HV
    W = O.weights(xyz, st, None, 6.0, types, dim=2, poly_deg=2, hv_k=4, hv_scale=-1e-3 * N ** -4.0)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(types, grid, 2)
    for t, w in W.items():
        der.setWeights(t, w)
    p = cosine_bell_setup()
    yield dict(xyz=xyz, st=st, W=W, grid=grid, der=der, p=p, h0=R.exact_cosine_bell(xyz))
    grid.close()


def _run(b, dtype, resident, steps, hv=True, arith=None, chunks=1):
    p = b["p"]
    pde = R.CosineBell(b["grid"], b["der"], p["a"], p["alpha"], p["T"], hv, dtype=dtype)
    if arith is not None:
        pde.setArithmetic(arith)
    else:
        pde.setShape(1, 256)
    pde.fillInitialConditions(b["h0"])
    for _ in range(chunks):
        pde.advance(R.RK4, p["dt"], steps // chunks, graph=not resident, resident=resident)
    out, t = pde.getLocalSolution(), pde.getTime()
    pde.close()
    return out, t


@pytest.mark.parametrize("dtype", [R.F64, R.F32])
@pytest.mark.parametrize("hv", [True, False])
def test_resident_cosine_bell_equals_one_lane_kernels(bell, dtype, hv):
    steps = 40
    res, t_res = _run(bell, dtype, True, steps, hv)
    ref, t_ref = _run(bell, dtype, False, steps, hv)
    assert np.array_equal(res, ref)
    assert t_res == t_ref
    assert np.array_equal(_run(bell, dtype, True, steps, hv, chunks=4)[0], res)
    if dtype == R.F64 and hv:
        p = bell["p"]
        cu, cv = O.cosine_bell_coeffs(bell["xyz"], a=p["a"], alpha=p["alpha"], u0=p["u0"])
        ora = O.rk4_advect(bell["st"], None, bell["W"][O.LAMBDA], bell["W"][O.THETA], bell["W"][O.HV], cu, cv,
                           bell["h0"], p["dt"], steps)
        assert np.array_equal(res, ora)


def test_resident_in_the_reference_arithmetic(bell):
    """Unfused (reference) arithmetic: the resident launch gives the plain
    path's bits."""
    steps = 20
    res, _ = _run(bell, R.F64, True, steps, arith=R.ARITH_UNFUSED)
    ref, _ = _run(bell, R.F64, False, steps, arith=R.ARITH_UNFUSED)
    assert np.array_equal(res, ref)


def test_resident_heat(ctx):
    N, n = 4096, 50
    xyz, st = sphere_problem(N, n, 2)
    W = O.weights(xyz, st, None, 0.25 / np.sqrt(4 * np.pi / N), O.LSFC, dim=2, poly_deg=3)[O.LSFC]
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(R.LSFC, grid, 2)
    der.setWeights(R.LSFC, W)
    u0 = R.exact_sph_heat(xyz, 8, np.random.default_rng(3).standard_normal(81), 0.0)
    outs = []
    for resident in (True, False):
        pde = R.HeatSphere(grid, der, 1.0, dtype=R.F64)
        pde.setShape(1, 256)
        pde.fillInitialConditions(u0)
        pde.advance(R.RK4, 1e-5, 25, resident=resident)
        outs.append(pde.getLocalSolution())
        pde.close()
    assert np.array_equal(outs[0], outs[1])
    assert np.array_equal(outs[0], O.rk4_heat(st, None, W, u0, 1e-5, 25))
    grid.close()


def test_resident_weights_in_shared_memory(ctx):
    """37-node stencils (10 chunks: no register-resident variant), so the
    weights stay in shared memory: FP64 advection equals the oracle bit for
    bit, FP32 with hyperviscosity equals the one-lane kernels."""
    N, n = 4096, 37
    xyz, st = sphere_problem(N, n, 6)
    types = O.LAMBDA | O.THETA | O.HV
    W = O.weights(xyz, st, None, 6.0, types, dim=2, poly_deg=2, hv_k=4, hv_scale=-1e-3 * N ** -4.0)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(types, grid, 2)
    for t, w in W.items():
        der.setWeights(t, w)
    p = cosine_bell_setup()
    b = dict(grid=grid, der=der, p=p, h0=R.exact_cosine_bell(xyz))
    res, _ = _run(b, R.F64, True, 20, hv=False)
    cu, cv = O.cosine_bell_coeffs(xyz, a=p["a"], alpha=p["alpha"], u0=p["u0"])
    assert np.array_equal(res, O.rk4_advect(st, None, W[O.LAMBDA], W[O.THETA], None, cu, cv, b["h0"], p["dt"], 20))
    res, _ = _run(b, R.F32, True, 20, hv=True)
    assert np.array_equal(res, _run(b, R.F32, False, 20, hv=True)[0])
    grid.close()


@pytest.mark.parametrize("N", [40, 1000, 2562])
def test_resident_small_and_ragged_grids(ctx, N):
    """N = 40: a cluster of 2 CTAs, the second with 8 rows; N = 1000: 16 CTAs
    of 64 rows, the last with 40; N = 2562: 16 CTAs of 192 rows, the last two
    without rows.  Equal to the oracle bit for bit."""
    n = 10
    xyz = R.fibonacci_nodes(N, 11)
    st = R.knn_stencils(xyz, n)
    W = O.weights(xyz, st, None, 2.0, O.LSFC, dim=2, poly_deg=1)[O.LSFC]
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(R.LSFC, grid, 2)
    der.setWeights(R.LSFC, W)
    u0 = np.cos(2 * xyz[:, 1]) + xyz[:, 0]
    pde = R.HeatSphere(grid, der, 1.0, dtype=R.F64)
    pde.fillInitialConditions(u0)
    pde.advance(R.RK4, 1e-3, 7, resident=True)
    out = pde.getLocalSolution()
    pde.close()
    assert np.array_equal(out, O.rk4_heat(st, None, W, u0, 1e-3, 7))
    grid.close()


def test_resident_refuses_large_grids_and_tracers(ctx):
    N, n = 40962, 31
    xyz = R.fibonacci_nodes(N, 4)
    st = R.knn_stencils(xyz, n)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(R.LSFC, grid, 2)
    der.setEpsilon(10.0)
    der.setPolynomialDegree(1)
    der.computeAllWeightsForAllStencils()
    pde = R.HeatSphere(grid, der, 1.0, dtype=R.F64)
    pde.fillInitialConditions(np.ones(N))
    with pytest.raises(R.RbffdError) as e:
        pde.advance(R.RK4, 1e-5, 2, resident=True)
    assert e.value.status == -5
    assert pde.getTime() == 0.0
    pde.close()
    grid.close()
    small = R.Grid(ctx, xyz[:1024], R.knn_stencils(xyz[:1024], 13))
    der = R.RBFFD(R.LSFC, small, 2)
    der.setEpsilon(4.0)
    der.setPolynomialDegree(1)
    der.computeAllWeightsForAllStencils()
    pde = R.HeatSphere(small, der, 1.0, dtype=R.F32, ntracers=4)
    pde.fillInitialConditions(np.ones((1024, 4)))
    with pytest.raises(R.RbffdError) as e:
        pde.advance(R.RK4, 1e-5, 2, resident=True)
    assert e.value.status == -5
    pde.close()
    small.close()
