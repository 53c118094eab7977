"""Vortex roll-up (VortexRollup::solve, src/pdes/hyperbolic/vortex_rollup.cpp:27-57;
ExactRollup, tests/experiments/vortex_rollup_on_sphere/exact_rollup.h) and the
solution norms of PDE::calcSolNorms (src/pdes/pde.cpp:467-510).

CPU: the norms equal the reference's own norms.cpp (compiled into oracle/_ref)
bit for bit, including the relative rule for exact norms <= 1e-10; w(theta)
and the exact roll-up equal the oracle's restatement bit for bit.
GPU: VortexRollup in FP64 (one lane per row) advances to the oracle's bits
with only the LAMBDA and HV weights computed; FP32 within 1e-5;
checkLocalError's norms are rbffd_sol_norms'."""
import numpy as np
import pytest

import oracle as O
import rbffd_gpu_b200 as R
from helpers import has_gpu, rel_l2


@pytest.mark.skipif(O.ref_lib("ref_norms") is None, reason="reference sources not built")
@pytest.mark.parametrize("case", ["random", "zero_exact", "tiny_exact", "empty", "single"])
def test_norms_equal_the_reference(case):
    rng = np.random.default_rng(3)
    n = {"empty": 0, "single": 1}.get(case, 5000)
    exact = rng.standard_normal(n)
    if case == "zero_exact":
        exact[:] = 0.0
    if case == "tiny_exact":
        exact *= 1e-14
    sol = exact + 1e-3 * rng.standard_normal(n)
    got = R.sol_norms(sol, exact)
    want = O.ref_sol_norms(sol, exact)
    assert [got[k] for k in R.api.NORM_NAMES] == list(want)


def test_vortex_coefficients_and_exact_solution():
    xyz = np.concatenate([R.fibonacci_nodes(5000, 2), [[0.0, 0.0, 1.0], [0.0, 0.0, -1.0], [1.0, 0.0, 0.0]]])
    w = R.vortex_rollup_coefficients(xyz)
    assert np.array_equal(w, O.vortex_rollup_w(xyz))
    assert w[-3] == 0.0 and w[-2] == 0.0  # the poles: rho = 3 cos(theta) ~ 0
    for t in (0.0, 0.7, 3.0):
        assert np.array_equal(R.exact_vortex_rollup(xyz, t), O.exact_vortex_rollup(xyz, t))


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a GPU")
def test_vortex_rollup_pde():
    N, n = 4096, 31
    xyz = R.fibonacci_nodes(N, 4)
    st = R.knn_stencils(xyz, n)
    types = O.LAMBDA | O.HV
    W = O.weights(xyz, st, None, 6.0, types, dim=2, poly_deg=2, hv_k=4, hv_scale=-1e-3 * N ** -4.0)
    ctx = R.Context(0)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(types, grid, 2)
    for t, w in W.items():
        der.setWeights(t, w)
    h0 = R.exact_vortex_rollup(xyz, 0.0)
    dt, steps = 0.01, 50  # RK4 stable: dt |lambda| ~ 0.8 for w D_lambda on this grid
    w = O.vortex_rollup_w(xyz)
    ref = O.rk4_advect(st, None, W[O.LAMBDA], W[O.LAMBDA], W[O.HV], w, np.zeros(N), h0, dt, steps)
    pde = R.VortexRollup(grid, der, True)
    pde.setShape(1, 256)
    pde.fillInitialConditions(h0)
    pde.advance(R.RK4, dt, steps)
    assert np.array_equal(pde.getLocalSolution(), ref)
    exact = R.exact_vortex_rollup(xyz, dt * steps)
    norms = pde.checkLocalError(exact)
    assert norms == R.sol_norms(pde.getLocalSolution(), exact)
    assert pde.checkGlobalError(exact) == norms
    assert pde.getLocalSolution(7) == pde.getLocalSolution()[7]
    pde.setStartEndTime(2.0, 3.0)
    assert pde.getTime() == 2.0
    assert norms["l2_rel"] < 0.1  # 3.7e-2 at t = 0.5: the roll-up steepens, n = 31 on 4096 nodes
    pde.close()
    p32 = R.VortexRollup(grid, der, True, dtype=R.F32)
    p32.fillInitialConditions(h0)
    p32.advance(R.RK4, dt, steps)
    assert rel_l2(p32.getLocalSolution(), ref) < 1e-5
    p32.close()
    grid.close()
    ctx.close()
