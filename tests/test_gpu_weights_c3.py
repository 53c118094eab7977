"""The batched weight configuration itself on the device: 10^6 stencils on
10^6 seeded Fibonacci nodes, n uniform over {17, 31, 50, 101} with polynomial
degree {1, 2, 3, 4} matched to n, eps ~ U[2, 8] per stencil, the tangential
gradients XSFC, YSFC, ZSFC (rbffd.cpp:465-489), solved in one persistent
launch.

At these shape parameters (eps h ~ 0.007-0.03) the saddle-point systems
reach condition numbers of 1e17-1e22, so weights are not compared entry by
entry.  The checks are the ones conditioning allows:
  * backward stability: each device solution of the device-assembled system
    has a relative residual below m * 2^-53 (LU with partial pivoting's
    guarantee; the oracle's own solutions of these systems stay below
    0.004 m 2^-53), and the stored weights are exactly that solution;
  * derivatives: on a sample of 2000 stencils the device weights and the
    oracle's (its own assembly and dgesv restatement) differentiate constants,
    x, y, z and a smooth field alike: within 1e-8, 1e-6 and 1e-3.  For scale,
    LAPACK's dgesv (numpy) on the oracle's own systems differs from the oracle
    by up to 7.6e-11, 1.6e-8 and 5.4e-5; the device's assembly differs from the
    oracle's by an ulp here and there (CUDA's exp, sin, cos against glibc's),
    which at these condition numbers moves constants' derivatives to ~1e-9.
The condition numbers per system size are printed.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
import rbffd_gpu_b200 as R
from rbffd_gpu_b200 import _lib

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

N = 1_000_000
SIZES, DEGS = (17, 31, 50, 101), (1, 2, 3, 4)
PSIZE = {1: 4, 2: 6, 3: 10, 4: 15}
TYPES = O.XSFC | O.YSFC | O.ZSFC


@pytest.fixture(scope="module")
def c3(ctx):
    xyz = R.fibonacci_nodes(N, 3)
    full = R.knn_stencils(xyz, max(SIZES))
    rng = np.random.default_rng(3)
    pick = rng.integers(0, len(SIZES), N)
    lens = np.array(SIZES, dtype=np.int32)[pick]
    degs = np.array(DEGS, dtype=np.int32)[pick]
    eps = rng.uniform(2.0, 8.0, N)
    grid = R.Grid(ctx, xyz, full, st_len=lens)
    der = R.RBFFD(R.XSFC | R.YSFC | R.ZSFC, grid, 2)
    der.setEpsilon(eps)
    der.setPolynomialDegree(1, deg_per_row=degs)
    der.computeAllWeightsForAllStencils()
    yield dict(xyz=xyz, full=full, lens=lens, degs=degs, eps=eps, grid=grid, der=der)
    grid.close()


def _assemble(grid, rows, degs, eps, m):
    out = np.zeros((len(rows), m, m + 3))
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    p = _lib.WeightParams(TYPES, 2, 1, 4, 0.0, 0.0)
    grid.ctx.check(grid.ctx.L.rbffd_weights_assemble(grid.h, ctypes.byref(p), eps.ctypes.data_as(_lib.dp), 0.0,
                                                     degs.ctypes.data_as(_lib.ip), rows.ctypes.data_as(_lib.ip),
                                                     len(rows), out.ctypes.data_as(_lib.dp)), "assemble")
    return out


def _gesv(ctx, A, B):
    batch, m, _ = A.shape
    dA = torch.tensor(A, dtype=torch.float64, device="cuda")
    dB = torch.tensor(B, dtype=torch.float64, device="cuda")
    info = torch.zeros(batch, dtype=torch.int32, device="cuda")
    ctx.check(ctx.L.rbffd_batched_gesv_dev(ctx.h, m, B.shape[2], batch, dA.data_ptr(), dB.data_ptr(),
                                           info.data_ptr()), "gesv")
    return dB.cpu().numpy(), info.cpu().numpy()


def test_c3_weights_are_backward_stable_solutions(ctx, c3):
    """Per system size, 48 stencils: the device-assembled systems solved by
    the device have relative residuals of LU's order, and the stored XSFC
    weights are exactly the first n entries of those solutions."""
    grid, degs, eps, lens = c3["grid"], c3["degs"], c3["eps"], c3["lens"]
    wx = c3["der"].getWeights(R.XSFC)
    for d, n in zip(DEGS, SIZES):
        rows = np.nonzero(degs == d)[0][::4000][:48]
        m = n + PSIZE[d]
        aug = _assemble(grid, rows, degs, eps, m)
        A, B = aug[:, :, :m], aug[:, :, m:]
        X, info = _gesv(ctx, A, B)
        assert (info == 0).all()
        Al, Xl, Bl = A.astype(np.longdouble), X.astype(np.longdouble), B.astype(np.longdouble)
        res = np.abs(np.einsum("bij,bjk->bik", Al, Xl) - Bl).max(axis=(1, 2))
        scale = np.abs(Al).sum(axis=2).max(axis=1) * np.abs(Xl).max(axis=(1, 2)) + np.abs(Bl).max(axis=(1, 2))
        rel = (res / scale).astype(np.float64)
        assert rel.max() <= m * 2.0 ** -53, (d, rel.max())
        kap = [np.linalg.cond(A[k]) for k in range(0, len(rows), 8)]
        print("m=%d: kappa median %.2e, max %.2e; relative residual max %.2e" % (m, np.median(kap), max(kap),
                                                                                  rel.max()))
        assert np.array_equal(wx[rows, :n], X[:, :n, 0])
        assert lens[rows].tolist() == [n] * len(rows)


def test_c3_derivatives_agree_with_the_oracle(c3):
    xyz, full, degs, eps, der = c3["xyz"], c3["full"], c3["degs"], c3["eps"], c3["der"]
    x, y, z = xyz.T
    funcs = {"one": (np.ones(N), 1e-8), "x": (x, 1e-6), "y": (y, 1e-6), "z": (z, 1e-6),
             "smooth": (np.sin(2 * x) * np.cos(3 * y) + z * z, 1e-3)}
    dev = {(t, k): der.applyWeightsForDeriv(t, f) for t in (R.XSFC, R.YSFC, R.ZSFC) for k, (f, _) in funcs.items()}
    S = np.arange(0, N, 500)
    worst = {}
    for d, n in zip(DEGS, SIZES):
        rows = S[degs[S] == d]
        W = O.weights(xyz, np.ascontiguousarray(full[rows][:, :n]), None, eps, TYPES, dim=2,
                      deg_per_row=degs[rows])
        for t in (O.XSFC, O.YSFC, O.ZSFC):
            for k, (f, tol) in funcs.items():
                orc = (W[t] * f[full[rows, :n]]).sum(axis=1)
                diff = float(np.abs(dev[(t, k)][rows] - orc).max())
                worst[(d, k)] = max(worst.get((d, k), 0.0), diff)
    print("device vs oracle, largest derivative differences per degree:",
          {"%d/%s" % key: "%.1e" % v for key, v in sorted(worst.items())})
    for (d, k), diff in worst.items():
        assert diff <= funcs[k][1], (d, k, diff)
