"""K2 parity: applyWeightsForDeriv on the device against the oracle's
restatement of RBFFD::applyWeightsForDeriv (rbffd.cpp:669-688).

The weights are the oracle's FP64 weights installed through
rbffd_weights_set, so the comparison isolates the SpMV:
* FP64 with one lane per row sums in the reference's order with fused
  multiply-adds: bit-exact.
* FP32 (FP32 weights, FP32 accumulation, rbffd_cl.cpp:669-682): relative L2
  error of the output against the FP64 result within ~ sqrt(n) * 2^-24 *
  sum|w u| / |sum w u|: 2e-6 for the first-derivative operators; 5e-5 for the
  Laplace-Beltrami operator, whose weights (~1/h^2, summing to zero) cancel by
  a factor of ~100 on a smooth field.
"""
import numpy as np
import pytest

import oracle as O
import rbffd_gpu_b200 as R
from tests.helpers import sphere_problem, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(ctx):
    N, n = 4096, 31
    xyz, st = sphere_problem(N, n, 1)
    types = O.LAMBDA | O.THETA | O.HV | O.LSFC
    W = O.weights(xyz, st, None, 0.035 * np.sqrt(N), types, dim=2, poly_deg=2, hv_k=4, hv_scale=-1e-3 * N ** -4.0)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(types, grid, 2)
    for t, w in W.items():
        der.setWeights(t, w)
    x, y, z = xyz.T
    u = np.exp(np.sin(2 * x) + np.cos(3 * y) * z) + 0.1 * x * y
    yield dict(xyz=xyz, st=st, W=W, grid=grid, der=der, u=u)
    grid.close()


@pytest.mark.parametrize("t", [O.LAMBDA, O.THETA, O.HV, O.LSFC])
def test_apply_fp64_bit_exact(setup, t):
    d = setup["der"].applyWeightsForDeriv(t, setup["u"], dtype=R.F64)
    ref = O.apply(setup["st"], None, setup["W"][t], setup["u"])
    assert np.array_equal(d, ref)


@pytest.mark.parametrize("t,tol", [(O.LAMBDA, 2e-6), (O.THETA, 2e-6), (O.LSFC, 5e-5)])
def test_apply_fp32_tolerance(setup, t, tol):
    d = setup["der"].applyWeightsForDeriv(t, setup["u"], dtype=R.F32)
    ref = O.apply(setup["st"], None, setup["W"][t], setup["u"])
    assert rel_l2(d, ref) < tol


def test_apply_subrange_writes_only_range(setup):
    u = setup["u"]
    out = np.full(len(u), -7.0)
    setup["der"].applyWeightsForDeriv(O.THETA, u, out, start_indx=1000, nb_stencils=500)
    ref = O.apply(setup["st"], None, setup["W"][O.THETA], u)
    assert np.array_equal(out[1000:1500], ref[1000:1500])
    assert (out[:1000] == -7.0).all() and (out[1500:] == -7.0).all()


def test_weights_roundtrip(setup):
    for t, w in setup["W"].items():
        assert np.array_equal(setup["der"].getWeights(t), w)


def test_apply_ragged_stencils(ctx):
    # stencils of different lengths: the padded ELL slots must contribute nothing
    N, n = 2562, 31
    xyz, st = sphere_problem(N, n, 5)
    rng = np.random.default_rng(0)
    lens = rng.integers(7, n + 1, size=N).astype(np.int32)
    W = O.weights(xyz, st, lens, 5.0, O.XSFC, dim=2, poly_deg=1)
    grid = R.Grid(ctx, xyz, st, st_len=lens)
    der = R.RBFFD(O.XSFC, grid, 2)
    der.setWeights(O.XSFC, W[O.XSFC])
    u = np.cos(xyz[:, 0] * 3) + xyz[:, 2]
    d = der.applyWeightsForDeriv(O.XSFC, u)
    assert np.array_equal(d, O.apply(st, lens, W[O.XSFC], u))
    grid.close()


@pytest.mark.parametrize("dtype", [R.F64, R.F32])
def test_apply_dev_multi_tracer_caller_order(setup, dtype):
    """Device-pointer apply on [N][T] data in the caller's node order."""
    torch = pytest.importorskip("torch")
    T = 3
    u = np.stack([setup["u"], np.cos(setup["u"]), setup["u"] ** 2], axis=1)
    tdt = torch.float64 if dtype == R.F64 else torch.float32
    du = torch.tensor(u, dtype=tdt, device="cuda")
    out = torch.zeros_like(du)
    setup["der"].applyWeightsForDerivDev(O.LSFC, du.data_ptr(), out.data_ptr(), dtype=dtype, ntracers=T)
    ref = O.apply(setup["st"], None, setup["W"][O.LSFC], u)
    got = out.double().cpu().numpy()
    if dtype == R.F64:
        assert np.array_equal(got, ref)
    else:
        assert rel_l2(got, ref) < 5e-5


def test_grid_rejects_bad_stencils(ctx):
    xyz, st = sphere_problem(2562, 17, 5)
    bad = st.copy()
    bad[10, 0] = 11  # centre not first (rbffd.cpp:916-928)
    with pytest.raises(R.RbffdError):
        R.Grid(ctx, xyz, bad)
    bad = st.copy()
    bad[5, 3] = 2562  # out of range
    with pytest.raises(R.RbffdError):
        R.Grid(ctx, xyz, bad)
