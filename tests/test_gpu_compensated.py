"""Compensated FP32 state (rbffd_pde_set_compensated_state): stage 3 adds
each RK4 increment with an exact two-sum and carries the lost rounding into
the next step, so long runs of small steps stay close to the FP64 result."""
import numpy as np
import pytest

import oracle as O
import rbffd_gpu_b200 as R
from tests.helpers import sphere_problem, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def heat4096(ctx):
    N, n = 4096, 50
    xyz, st = sphere_problem(N, n, 6)
    W = O.weights(xyz, st, None, 0.25 / np.sqrt(4 * np.pi / N), O.LSFC, dim=2, poly_deg=3)[O.LSFC]
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(R.LSFC, grid, 2)
    der.setWeights(R.LSFC, W)
    u0 = R.exact_sph_heat(xyz, 10, np.random.default_rng(3).standard_normal(121), 0.0)
    yield dict(grid=grid, der=der, u0=u0, N=N)
    grid.close()


def _run(h, dtype, steps, dt, comp=False, shape=None, ntr=1, graph=True, u0=None):
    pde = R.HeatSphere(h["grid"], h["der"], 1.0, dtype=dtype, ntracers=ntr)
    if comp:
        pde.setCompensatedState(True)
    if shape == "tile":
        pde.setTiledShape(128, 1)
    elif shape is not None:
        pde.setShape(*shape)
    pde.fillInitialConditions(h["u0"] if u0 is None else u0)
    pde.advance(R.RK4, dt, steps, graph=graph)
    out = pde.getLocalSolution()
    pde.close()
    return out


@pytest.mark.parametrize("shape", [(1, 128), "tile", None])
def test_compensated_fp32_stays_near_fp64(heat4096, shape):
    """2000 heat steps of 1e-6 (each moves u by about 1e-4 of itself): the
    plain FP32 state drifts 1.6e-6 from FP64, the compensated one stays within
    2e-7, whatever the stage kernel (one lane per row, a halo tile, the
    autotuned shape)."""
    dt, steps = 1e-6, 2000
    ref = _run(heat4096, R.F64, steps, dt, shape=(1, 128))
    plain = _run(heat4096, R.F32, steps, dt, shape=shape)
    comp = _run(heat4096, R.F32, steps, dt, comp=True, shape=shape)
    assert rel_l2(comp, ref) < 2e-7
    assert rel_l2(plain, ref) > 5 * rel_l2(comp, ref)


def test_compensated_multi_tracer_and_unfused_path(heat4096):
    """Four tracers on the tiled kernel, and the unfused path (separate apply
    and update launches): each within 2e-7 of FP64."""
    dt, steps = 1e-6, 1500
    rng = np.random.default_rng(9)
    u4 = heat4096["u0"][:, None] * (1.0 + 0.1 * rng.random((1, 4)))
    ref = _run(heat4096, R.F64, steps, dt, shape=(1, 128), ntr=4, u0=u4)
    comp = _run(heat4096, R.F32, steps, dt, comp=True, shape="tile", ntr=4, u0=u4)
    assert rel_l2(comp, ref) < 2e-7
    ref1 = _run(heat4096, R.F64, 300, dt, shape=(1, 128))
    pde = R.HeatSphere(heat4096["grid"], heat4096["der"], 1.0, dtype=R.F32)
    pde.setCompensatedState(True)
    pde.fillInitialConditions(heat4096["u0"])
    pde.advance(R.RK4, dt, 300, unfused=True)
    assert rel_l2(pde.getLocalSolution(), ref1) < 1e-7
    pde.close()


def test_compensated_state_is_cleared_by_set_state_and_switches_off(heat4096):
    """A second run from the same initial state gives the first run's bits
    (set_state clears the correction); switching it off returns the plain
    FP32 bits; FP64 PDEs and the cluster-resident path refuse it."""
    dt, steps = 1e-6, 200
    pde = R.HeatSphere(heat4096["grid"], heat4096["der"], 1.0, dtype=R.F32)
    pde.setShape(1, 128)
    pde.setCompensatedState(True)
    outs = []
    for _ in range(2):
        pde.fillInitialConditions(heat4096["u0"])
        pde.advance(R.RK4, dt, steps, graph=True)
        outs.append(pde.getLocalSolution())
    assert np.array_equal(outs[0], outs[1])
    with pytest.raises(R.RbffdError) as e:
        pde.advance(R.RK4, dt, 2, resident=True)
    assert e.value.status == -5
    pde.setCompensatedState(False)
    pde.fillInitialConditions(heat4096["u0"])
    pde.advance(R.RK4, dt, steps, graph=True)
    assert np.array_equal(pde.getLocalSolution(), _run(heat4096, R.F32, steps, dt, shape=(1, 128)))
    pde.close()
    p64 = R.HeatSphere(heat4096["grid"], heat4096["der"], 1.0, dtype=R.F64)
    with pytest.raises(R.RbffdError) as e:
        p64.setCompensatedState(True)
    assert e.value.status == -5
    p64.close()
