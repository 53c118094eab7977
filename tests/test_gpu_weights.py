"""K1 parity: batched FP64 weights on the device against the oracle's
restatement of RBFFD::computeAllWeightsForStencil_Direct (rbffd.cpp:225-352).

The chain, step by step:
1. assembly -- every entry of the device-built [A | B] within a few ulp of the
   oracle's (the difference is CUDA's vs glibc's exp/sin/cos/atan2);
2. elimination -- on identical systems the device solver's result equals the
   oracle's dgesv restatement bit for bit;
3. weights -- within a bound set by the conditioning of the systems (RBF-FD
   saddle-point systems reach kappa ~ 1e13-1e15 here, so one-ulp input
   differences move weights by up to ~kappa * 1e-16), and the derivatives
   they produce agree with the oracle's and with the exact derivative.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
import rbffd_gpu_b200 as R
from rbffd_gpu_b200 import _lib
from tests.helpers import sphere_problem, rel_l2

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _params(types, dim=2, deg=0, hv_k=4, hv_gamma=0.0, hv_nodes=0.0):
    return _lib.WeightParams(types, dim, deg, hv_k, hv_gamma, hv_nodes)


def _device_assemble(grid, types, deg, eps, rows, dim=2, hv_k=4):
    K = bin(types).count("1")
    n = grid.n_pad
    m = n + O.lib().orc_poly_size(deg)
    out = np.zeros((len(rows), m, m + K))
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    epsv = np.full(grid.N, eps)
    p = _params(types, dim, deg, hv_k)
    grid.ctx.check(grid.ctx.L.rbffd_weights_assemble(grid.h, ctypes.byref(p), epsv.ctypes.data_as(_lib.dp), 0.0, None,
                                                     rows.ctypes.data_as(_lib.ip), len(rows),
                                                     out.ctypes.data_as(_lib.dp)), "assemble")
    return out


@pytest.mark.parametrize("N,n,deg,eps,types", [
    (4096, 31, 0, 2.24, O.LAMBDA | O.THETA | O.HV),
    (4096, 31, 2, 2.24, O.LAMBDA | O.THETA | O.HV),
    (10242, 50, 3, 0.044 * np.sqrt(10242) - 0.14, O.LSFC),
    (10242, 17, 1, 4.0, O.XSFC | O.YSFC | O.ZSFC),
    (2562, 101, 4, 9.0, O.XSFC | O.YSFC | O.ZSFC | O.LAPL | O.INTERP),
])
def test_assembly_matches_oracle(ctx, N, n, deg, eps, types):
    xyz, st = sphere_problem(N, n, 1)
    grid = R.Grid(ctx, xyz, st)
    rows = list(range(0, N, max(1, N // 37)))
    dev = _device_assemble(grid, types, deg, eps, rows)
    ulps = []
    for k, r in enumerate(rows):
        ref = O.assemble(xyz, st[r], deg, eps, types, dim=2, hv_k=4)
        # Entries such as x0 (x0.xj) - xj (rbffd.cpp:465-489) or cos(th_j) sin(lam_i - lam_j)
        # are differences of nearly equal terms near the centre, so their rounding is
        # relative to the size of the column, not of the entry.
        col_scale = np.maximum(np.abs(ref).max(axis=0), 1e-300)
        err = np.abs(dev[k] - ref)
        assert (err <= 1e-13 * col_scale[None, :]).all(), (r, (err / col_scale).max())
        nz = ref != 0
        ulps.append(np.median(err[nz] / (np.abs(ref[nz]) * 2.0 ** -52)))
    assert np.median(ulps) <= 2.0  # typical entries agree to within two ulp
    grid.close()


def _gesv_dev(ctx, A, B):
    batch, m, _ = A.shape
    nrhs = B.shape[2]
    dA = torch.tensor(A, dtype=torch.float64, device="cuda")
    dB = torch.tensor(B, dtype=torch.float64, device="cuda")
    info = torch.zeros(batch, dtype=torch.int32, device="cuda")
    ctx.check(ctx.L.rbffd_batched_gesv_dev(ctx.h, m, nrhs, batch, dA.data_ptr(), dB.data_ptr(), info.data_ptr()),
              "gesv")
    return dB.cpu().numpy(), info.cpu().numpy()


@pytest.mark.parametrize("deg", [0, 2, 3])
def test_elimination_bit_exact_on_identical_systems(ctx, deg):
    xyz, st = sphere_problem(4096, 31, 1)
    systems = [O.assemble(xyz, st[r], deg, 2.24, O.LAMBDA | O.THETA | O.HV) for r in range(0, 4096, 64)]
    m = systems[0].shape[0]
    A = np.stack([s[:, :m] for s in systems])
    B = np.stack([s[:, m:] for s in systems])
    X, info = _gesv_dev(ctx, A, B)
    assert (info == 0).all()
    for k in range(len(systems)):
        assert np.array_equal(X[k], O.lu_solve(A[k], B[k]))


# sizes that reach each elimination: row swaps (m <= 40), a row map (41-96), blocked (> 96)
@pytest.mark.parametrize("m,nrhs", [(1, 1), (7, 2), (32, 3), (33, 1), (41, 3), (67, 1), (96, 2), (100, 4), (126, 3),
                                    (160, 2)])
def test_elimination_bit_exact_random(ctx, m, nrhs):
    rng = np.random.default_rng(m)
    A = rng.normal(size=(9, m, m))
    B = rng.normal(size=(9, m, nrhs))
    X, info = _gesv_dev(ctx, A, B)
    assert (info == 0).all()
    for k in range(9):
        assert np.array_equal(X[k], O.lu_solve(A[k], B[k]))


@pytest.mark.parametrize("m,col", [(6, 3), (60, 45), (116, 8)])
def test_elimination_reports_zero_pivot(ctx, m, col):
    """A zero pivot column, in the unblocked (m <= 40) and the blocked
    elimination (a panel's first and a later column)."""
    A = np.eye(m)[None].repeat(2, axis=0)
    A[1, :, col] = 0.0  # column `col` exactly zero: zero pivot at that step
    B = np.ones((2, m, 1))
    _, info = _gesv_dev(ctx, A, B)
    assert info[0] == 0 and info[1] == col + 1


def test_weights_match_oracle_cosine_bell_setup(ctx):
    N, n = 4096, 31
    xyz, st = sphere_problem(N, n, 1)
    types = O.LAMBDA | O.THETA | O.HV
    eps = 0.035 * np.sqrt(N)
    grid = R.Grid(ctx, xyz, st)
    for deg in (0, 2):
        der = R.RBFFD(types, grid, 2)
        der.setEpsilon(eps)
        der.setHVScalars(4, 1e-3)
        der.setPolynomialDegree(deg)
        der.computeAllWeightsForAllStencils()
        W = O.weights(xyz, st, None, eps, types, dim=2, poly_deg=deg, hv_k=4, hv_scale=der.getHVScalar())
        x, y, z = xyz.T
        f = np.exp(np.sin(2 * x) + np.cos(3 * y) * z)
        for t in (O.LAMBDA, O.THETA, O.HV):
            wg = der.getWeights(t)
            # kappa ~ 1e14 here (see module docstring): weights agree to ~1e-3, derivatives much closer
            assert rel_l2(wg, W[t]) < 5e-3, (deg, t)
            dg = O.apply(st, None, wg, f)
            do = O.apply(st, None, W[t], f)
            assert rel_l2(dg, do) < 1e-6, (deg, t)
    grid.close()


def test_weights_mixed_sizes_bucketed(ctx):
    """Mixed stencil sizes and polynomial degrees in one call (the batched
    configuration): n in {17,31,50,101}, degree matched {1,2,3,4}."""
    N = 6000
    xyz = R.fibonacci_nodes(N, 3)
    full = R.knn_stencils(xyz, 101)
    rng = np.random.default_rng(3)
    sizes = np.array([17, 31, 50, 101])
    pick = rng.integers(0, 4, N)
    lens = sizes[pick].astype(np.int32)
    degs = (pick + 1).astype(np.int32)
    eps = rng.uniform(10.0, 16.0, N)  # kappa moderate on this node count
    types = O.XSFC | O.YSFC | O.ZSFC
    grid = R.Grid(ctx, xyz, full, st_len=lens)
    der = R.RBFFD(types, grid, 2)
    der.setEpsilon(eps)
    der.setPolynomialDegree(1, deg_per_row=degs)
    der.computeAllWeightsForAllStencils()
    W = O.weights(xyz, full, lens, eps, types, dim=2, deg_per_row=degs)
    x, y, z = xyz.T
    f = np.sin(2 * x + y) * np.cos(z)
    for t in (O.XSFC, O.YSFC, O.ZSFC):
        wg = der.getWeights(t)
        for k in range(4):
            rows = pick == k
            assert np.all(wg[rows][:, sizes[k]:] == 0.0)
        assert rel_l2(O.apply(full, lens, wg, f), O.apply(full, lens, W[t], f)) < 1e-6
    grid.close()


def test_alt_sfc_operators(ctx):
    """ALT_XSFC/YSFC/ZSFC: asking for one computes X, Y, Z and all three
    (RBFFD::adjustForSFCTypes), and their weights are the oracle's projection
    of the device's X, Y, Z weights bit for bit (rbffd.cpp:337-347); on a
    smooth function they approximate the tangential gradient XSFC does."""
    N, n = 4096, 31
    xyz, st = sphere_problem(N, n, 3)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(R.ALT_YSFC | R.XSFC, grid, 2)
    der.setEpsilon(0.3 * np.sqrt(N))
    der.setPolynomialDegree(2)
    der.computeAllWeightsForAllStencils()
    assert der.computedTypes & (R.X | R.Y | R.Z | R.ALT_XSFC | R.ALT_ZSFC) == (R.X | R.Y | R.Z | R.ALT_XSFC | R.ALT_ZSFC)
    wx, wy, wz = (der.getWeights(t) for t in (R.X, R.Y, R.Z))
    want = O.alt_sfc(xyz, wx, wy, wz)
    for t, w in zip((R.ALT_XSFC, R.ALT_YSFC, R.ALT_ZSFC), want):
        assert np.array_equal(der.getWeights(t), w)
    f = np.exp(xyz[:, 0]) * np.sin(2 * xyz[:, 1])
    a = der.applyWeightsForDeriv(R.ALT_XSFC, f)
    b = der.applyWeightsForDeriv(R.XSFC, f)
    assert rel_l2(a, b) < 1e-2
    grid.close()


METHODS = (R.ELIM_AUTO, R.ELIM_UNBLOCKED, R.ELIM_BLOCKED, R.ELIM_ROW_MAP, R.ELIM_REGISTERS)


def _weights_by_method(ctx, xyz, full, lens, degs, eps, types, methods=METHODS):
    grid = R.Grid(ctx, xyz, full, st_len=lens)
    out = {}
    try:
        for meth in methods:
            ctx.setWeightsElimination(meth)
            assert ctx.getWeightsElimination() == meth
            der = R.RBFFD(types, grid, 2)
            der.setEpsilon(eps)
            der.setPolynomialDegree(1, deg_per_row=degs)
            der.computeAllWeightsForAllStencils()
            out[meth] = {t: der.getWeights(t) for t in (R.XSFC, R.YSFC, R.ZSFC)}
    finally:
        ctx.setWeightsElimination(R.ELIM_AUTO)
        grid.close()
    return out


def test_weights_every_elimination_same_bits(ctx):
    """The batched mix (n in {17, 31, 50, 101}, degrees 1-4: m = 21, 37, 60,
    116) solved with each elimination -- shared-memory unblocked, blocked
    panels, row map, and the rows held in registers -- gives the same weights
    bit for bit, and they differentiate like the oracle's."""
    N = 6000
    xyz = R.fibonacci_nodes(N, 5)
    full = R.knn_stencils(xyz, 101)
    rng = np.random.default_rng(5)
    sizes = np.array([17, 31, 50, 101])
    pick = rng.integers(0, 4, N)
    lens = sizes[pick].astype(np.int32)
    degs = (pick + 1).astype(np.int32)
    eps = rng.uniform(10.0, 16.0, N)
    types = R.XSFC | R.YSFC | R.ZSFC
    W = _weights_by_method(ctx, xyz, full, lens, degs, eps, types)
    for meth in METHODS[1:]:
        for t in (R.XSFC, R.YSFC, R.ZSFC):
            assert np.array_equal(W[meth][t], W[R.ELIM_AUTO][t]), (meth, t)
    Wo = O.weights(xyz, full, lens, eps, O.XSFC | O.YSFC | O.ZSFC, dim=2, deg_per_row=degs)
    f = np.sin(2 * xyz[:, 0] + xyz[:, 1]) * np.cos(xyz[:, 2])
    for t in (R.XSFC, R.YSFC, R.ZSFC):
        assert rel_l2(O.apply(full, lens, W[R.ELIM_REGISTERS][t], f), O.apply(full, lens, Wo[t], f)) < 1e-6


@pytest.mark.parametrize("n,deg", [(110, 4), (51, 3)])
def test_register_elimination_at_its_size_limits(ctx, n, deg):
    """The register-resident shapes at their largest systems: m = 125 with
    three right-hand sides fills 4 column chunks of 16 warps x 8 rows exactly
    (m + K = 128); m = 61 fills the 8-warp shape's 2 chunks (m + K = 64).
    Same bits as the shared-memory elimination."""
    N = 3000
    xyz = R.fibonacci_nodes(N, 6)
    full = R.knn_stencils(xyz, n)
    lens = np.full(N, n, dtype=np.int32)
    degs = np.full(N, deg, dtype=np.int32)
    eps = np.random.default_rng(6).uniform(8.0, 12.0, N)
    W = _weights_by_method(ctx, xyz, full, lens, degs, eps, R.XSFC | R.YSFC | R.ZSFC,
                           methods=(R.ELIM_UNBLOCKED, R.ELIM_REGISTERS))
    for t in (R.XSFC, R.YSFC, R.ZSFC):
        assert np.isfinite(W[R.ELIM_REGISTERS][t]).all()
        assert np.array_equal(W[R.ELIM_REGISTERS][t], W[R.ELIM_UNBLOCKED][t]), t


@pytest.mark.parametrize("meth", METHODS[1:])
def test_weights_singular_stencil_reported(ctx, meth):
    """A stencil that lists a node twice has two equal rows: every
    elimination meets an exactly zero pivot and the call reports it."""
    N, n = 2048, 31
    xyz = R.fibonacci_nodes(N, 7)
    st = R.knn_stencils(xyz, n)
    st[100, 7] = st[100, 6]
    grid = R.Grid(ctx, xyz, st)
    ctx.setWeightsElimination(meth)
    try:
        der = R.RBFFD(R.XSFC, grid, 2)
        der.setEpsilon(10.0)
        der.setPolynomialDegree(2)
        with pytest.raises(R.RbffdError):
            der.computeAllWeightsForAllStencils()
    finally:
        ctx.setWeightsElimination(R.ELIM_AUTO)
        grid.close()
