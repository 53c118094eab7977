"""Eigenvalue stability check (RBFFD::computeEigenvalues, src/rbffd/rbffd.cpp:703-873).

CPU: the library's classification (rbffd_eig_classify) equals the oracle's
restatement of the reference loop, including its start-from-|Re(eig(0))|
extremes and the 1e-8 zero band, and the entry points reject bad arguments.
GPU: every eigenvalue of the dense operator assembled on the device from the
grid's weights equals LAPACK dgeev's (numpy) on the oracle's dense matrix of
the same weights, within 1e-9 of the spectral radius as sets, and the counts
match."""
import ctypes

import numpy as np
import pytest

import oracle as O
import rbffd_gpu_b200 as R
from rbffd_gpu_b200 import _lib
from helpers import has_gpu


def _cases():
    rng = np.random.default_rng(11)
    yield np.array([3.0])
    yield np.array([-2.0, 1e-9, -1e-9, 5e-9, 0.0])
    yield np.array([1e-8, -1e-8, 1.0000001e-8, -1.0000001e-8])  # the band's edges
    yield np.array([-7.0, 4.0, 2.0, -1.0])        # first eigenvalue negative: max_pos starts at 7
    yield np.array([5.0, -1.0, -3.0])              # first positive: min_neg starts at 5
    yield np.array([-0.0, np.nextafter(0, 1)])
    for _ in range(20):
        n = int(rng.integers(1, 300))
        x = rng.standard_normal(n) * 10.0 ** rng.uniform(-10, 3, n)
        yield x


@pytest.mark.parametrize("re", list(_cases()))
def test_classification_equals_reference_loop(re):
    got, ret = R.eig_classify(re)
    want, want_ret = O.eig_classify(re)
    assert got == want
    assert ret == want_ret


def test_classification_tolerance_argument():
    re = np.array([-1e-6, 1e-6, 0.0, -2.0])
    got, _ = R.eig_classify(re, zero_tol=1e-5)
    assert (got["nb_zero"], got["nb_negative"], got["nb_positive"]) == (3, 1, 0)
    assert got == O.eig_classify(re, zero_tol=1e-5)[0]


def test_bad_arguments_rejected():
    L = _lib.load()
    o = _lib.EigOutput()
    one = np.ones(1)
    assert L.rbffd_eig_classify(None, 1, 1e-8, ctypes.byref(o), None) == -1
    assert L.rbffd_eig_classify(one.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0, 1e-8, None, None) == -1
    assert L.rbffd_eig_classify(one.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1, -1.0, None, None) == -1
    assert L.rbffd_eigenvalues(None, R.LSFC, 0, None, None, None, None) == -1


def _set_distance(a, b):
    """Largest distance from a point of either set to the other set."""
    d = np.abs(a[:, None] - b[None, :])
    return max(d.min(axis=1).max(), d.min(axis=0).max())


def _band(re, tol=1e-8):
    a = np.abs(re)
    return int(np.sum((a > tol / 10) & (a < tol * 10)))


def _check_against_oracle(der, which, N, st, w_hv=None, counts=True):
    lam_max, ev = der.computeEigenvalues(which, return_eigenvalues=True)
    res = der.cachedEigenvalues
    w = der.getWeights(which)
    A = O.dense_operator(st, None, w, w_hv)
    ref = O.eigenvalues(A)
    rho = np.abs(ref).max()
    assert ev.shape == (N,)
    assert _set_distance(ev, ref) <= 1e-9 * rho
    want, want_ret = O.eig_classify(ref.real)
    # the classification of the device's own eigenvalues is the reference loop's
    assert (res, lam_max) == O.eig_classify(ev.real)
    if counts:
        slack = _band(ref.real)
        for k in ("nb_positive", "nb_negative", "nb_zero"):
            assert abs(res[k] - want[k]) <= slack, (k, res, want)
    return res, ref


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a GPU")
def test_dense_eigenvalues_match_lapack_heat_operator():
    N, n = 1024, 31
    ctx = R.Context(0)
    xyz = R.fibonacci_nodes(N, 2)
    st = R.knn_stencils(xyz, n)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(R.LSFC, grid, 2)
    der.setEpsilon(0.3 * np.sqrt(N))
    der.setPolynomialDegree(2)
    der.computeAllWeightsForAllStencils()
    res, ref = _check_against_oracle(der, R.LSFC, N, st)
    # a Laplace-Beltrami operator: mostly negative spectrum, the constant mode near zero
    assert res["nb_negative"] >= 0.9 * N
    grid.close()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a GPU")
def test_dense_eigenvalues_match_lapack_advection_with_hyperviscosity():
    N, n = 1024, 31
    ctx = R.Context(0)
    xyz = R.fibonacci_nodes(N, 1)
    st = R.knn_stencils(xyz, n)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(R.LAMBDA | R.THETA, grid, 2)
    der.setUseHyperviscosity(1)
    der.setHVScalars(4, 1e-3)
    der.setEpsilon(6.0)
    der.setPolynomialDegree(2)
    der.computeAllWeightsForAllStencils()
    w_hv = der.getWeights(R.HV)
    _check_against_oracle(der, R.LAMBDA, N, st, w_hv=w_hv, counts=False)
    # without hyperviscosity: the plain operator
    der.setUseHyperviscosity(0)
    _check_against_oracle(der, R.THETA, N, st, counts=False)
    grid.close()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a GPU")
def test_eigenvalue_errors():
    ctx = R.Context(0)
    xyz = R.fibonacci_nodes(400, 3)
    st = R.knn_stencils(xyz, 17)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(R.LSFC, grid, 2)
    with pytest.raises(R.RbffdError) as e:  # weights not computed
        der.computeEigenvalues(R.LSFC)
    assert e.value.status == -6
    der.setEpsilon(4.0)
    der.computeAllWeightsForAllStencils()
    der.setUseHyperviscosity(1)
    with pytest.raises(R.RbffdError) as e:  # HV weights missing
        der.computeEigenvalues(R.LSFC)
    assert e.value.status == -6
    der.setUseHyperviscosity(0)
    assert ctx.L.rbffd_eigenvalues(grid.h, R.LSFC | R.LAMBDA, 0, None, None, None, None) == -1
    assert der.computeEigenvalues(R.LSFC) > 0
    grid.close()
    big = R.fibonacci_nodes(R_EIG_MAX + 1, 3)
    g2 = R.Grid(ctx, big, R.knn_stencils(big, 5))
    assert ctx.L.rbffd_eigenvalues(g2.h, R.LSFC, 0, None, None, None, None) == -5
    g2.close()
    ctx.close()


R_EIG_MAX = 16384


def test_hessenberg_eigenvalues_match_lapack():
    """The Arnoldi check's projected eigenproblem (host, shifted QR in complex
    arithmetic) against LAPACK (numpy) on random Hessenberg matrices of the
    sizes the check uses, scaled and shifted."""
    rng = np.random.default_rng(5)
    for n in (1, 2, 3, 8, 40, 64, 120):
        for trial in range(6):
            H = np.triu(rng.standard_normal((n, n)), -1) * 10.0 ** rng.uniform(-6, 6)
            ev, ref = R.hessenberg_eigenvalues(H), np.linalg.eigvals(H)
            assert _set_distance(ev, ref) <= 1e-10 * max(np.abs(ref).max(), 1e-300), (n, trial)
    with pytest.raises(R.RbffdError):
        R.hessenberg_eigenvalues(np.zeros((0, 0)))


def _rightmost_case(ctx, N, n, types, eps, deg, hv):
    xyz = R.fibonacci_nodes(N, 1)
    st = R.knn_stencils(xyz, n)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(types, grid, 2)
    if hv:
        der.setUseHyperviscosity(1)
        der.setHVScalars(4, 1e-3)
    der.setEpsilon(eps)
    der.setPolynomialDegree(deg)
    der.computeAllWeightsForAllStencils()
    return grid, der


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a GPU")
@pytest.mark.parametrize("case", ["advection_hv", "heat"])
def test_rightmost_eigenvalues_match_the_dense_check(case):
    """Arnoldi on the sparse operator against every eigenvalue of the dense
    check: the rightmost Ritz values equal the rightmost eigenvalues to 1e-7
    of the spectral radius, and the stability verdict (sign of the largest
    real part beyond the 1e-8 band) agrees."""
    ctx = R.Context(0)
    if case == "advection_hv":  # unstable: positive real parts (the cosine bell at eps = 6)
        grid, der = _rightmost_case(ctx, 4096, 31, R.LAMBDA, 6.0, 2, True)
        which, nev = R.LAMBDA, 5
    else:  # stable: the constant mode at 0, the rest negative
        grid, der = _rightmost_case(ctx, 2562, 31, R.LSFC, 0.25 * np.sqrt(2562 / (4 * np.pi)), 2, False)
        which, nev = R.LSFC, 4
    _, dense = der.computeEigenvalues(which, return_eigenvalues=True)
    dense = dense[np.argsort(-dense.real)]
    rho = np.abs(dense).max()
    out = der.computeRightmostEigenvalues(which, nev=nev, ncv=40, tol=1e-9)
    ev = out["eigenvalues"]
    assert out["nconv"] >= nev - 1, out
    top = ev[:nev - 1]  # the last wanted value may sit in a cluster; the others are pinned
    # every Ritz value is an eigenvalue of the dense check
    assert np.abs(top[:, None] - dense[None, :]).min(axis=1).max() <= 1e-7 * rho, (top, dense[:nev + 1])
    assert abs(ev[0].real - dense[0].real) <= 1e-7 * rho
    assert (ev[0].real > 1e-8) == (dense[0].real > 1e-8)
    grid.close()
    ctx.close()
