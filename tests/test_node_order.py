"""Node orders (the reordering step before the SpMV: the reference's
tests/util/cuthill_mckee/{main.cpp,reorder.h}).

CPU: rbffd_node_order equals the oracle's restatements -- the Morton curve and
reverse Cuthill-McKee with the reference utility's start-node search -- node
for node, on sphere grids with full and ragged stencils and on a graph with
several components; every order is a permutation; RCM narrows the stencil
graph's bandwidth as much as scipy's reverse Cuthill-McKee does (within 25%).
GPU: grids stored in the Morton, RCM and caller's orders advance the heat
equation to the oracle's FP64 bits (the order moves rows, never their
arithmetic)."""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.csgraph import reverse_cuthill_mckee

import oracle as O
import rbffd_gpu_b200 as R
from helpers import has_gpu


def _bandwidth(st, order, st_len=None):
    pos = np.empty(len(order), dtype=np.int64)
    pos[order] = np.arange(len(order))
    N, n = st.shape
    lens = np.full(N, n) if st_len is None else st_len
    return max(int(np.abs(pos[st[i, :lens[i]]] - pos[i]).max()) for i in range(N))


def _cases():
    for N, n, seed in ((500, 9, 1), (2562, 31, 2), (4000, 17, 3)):
        xyz = R.fibonacci_nodes(N, seed)
        yield f"sphere{N}_{n}", xyz, R.knn_stencils(xyz, n), None
    xyz = R.fibonacci_nodes(1500, 4)
    st = R.knn_stencils(xyz, 21)
    lens = np.random.default_rng(4).integers(1, 22, 1500).astype(np.int32)
    yield "ragged1500", xyz, st, lens
    # two separate clusters and isolated nodes: several components
    a = R.fibonacci_nodes(300, 5)
    xyz = np.concatenate([a, a + 10.0, [[50.0, 0, 0], [60.0, 0, 0]]])
    st = R.knn_stencils(xyz, 7)
    lens = np.full(len(xyz), 7, dtype=np.int32)
    lens[-2:] = 1
    yield "components", xyz, st, lens


CASES = list(_cases())


@pytest.mark.parametrize("name,xyz,st,lens", CASES, ids=[c[0] for c in CASES])
def test_orders_equal_the_oracle(name, xyz, st, lens):
    m = R.node_order(R.ORDER_MORTON, xyz=xyz)
    assert np.array_equal(m, O.morton_order(xyz))
    r = R.node_order(R.ORDER_RCM, stencils=st, st_len=lens)
    assert np.array_equal(r, O.rcm_order(st, lens))
    g = R.node_order(R.ORDER_GIVEN, xyz=xyz)
    assert np.array_equal(g, np.arange(len(xyz)))
    for o in (m, r):
        assert np.array_equal(np.sort(o), np.arange(len(xyz)))


@pytest.mark.parametrize("N,n", [(2562, 31), (10242, 50)])
def test_rcm_bandwidth_matches_scipy(N, n):
    xyz = R.fibonacci_nodes(N, 7)
    st = R.knn_stencils(xyz, n)
    rows = np.repeat(np.arange(N), n)
    A = sp.csr_matrix((np.ones(N * n), (rows, st.ravel())), shape=(N, N))
    A = ((A + A.T) > 0).astype(np.float64).tocsr()
    ref = reverse_cuthill_mckee(A, symmetric_mode=True)
    ours = R.node_order(R.ORDER_RCM, stencils=st)
    bw_ours, bw_ref = _bandwidth(st, ours), _bandwidth(st, ref)
    assert bw_ours <= 1.25 * bw_ref
    # against an unordered numbering (Fibonacci nodes come along a spiral in z,
    # already banded): the nodes relabelled at random
    p = np.random.default_rng(8).permutation(N)
    inv = np.empty(N, dtype=np.int64)
    inv[p] = np.arange(N)
    st_rand = inv[st[p]].astype(np.int32)
    assert _bandwidth(st_rand, R.node_order(R.ORDER_RCM, stencils=st_rand)) < _bandwidth(st_rand, np.arange(N)) / 5


def test_bad_arguments():
    xyz = R.fibonacci_nodes(50, 1)
    st = R.knn_stencils(xyz, 5)
    with pytest.raises(R.RbffdError):
        R.node_order(7, xyz=xyz)
    with pytest.raises(R.RbffdError):
        R.node_order(R.ORDER_MORTON, stencils=st)  # no coordinates
    bad = st.copy()
    bad[3, 2] = 50
    with pytest.raises(R.RbffdError):
        R.node_order(R.ORDER_RCM, stencils=bad)


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a GPU")
def test_every_order_gives_the_oracle_bits():
    N, n = 4096, 31
    xyz = R.fibonacci_nodes(N, 2)
    st = R.knn_stencils(xyz, n)
    h = np.sqrt(4 * np.pi / N)
    W = O.weights(xyz, st, None, 0.25 / h, O.LSFC, dim=2, poly_deg=2)[O.LSFC]
    u0 = R.exact_sph_heat(xyz, 8, np.random.default_rng(3).standard_normal(81), 0.0)
    ref = O.rk4_heat(st, None, W, u0, 1e-5, 12)
    ctx = R.Context(0)
    outs = {}
    for order in (R.ORDER_MORTON, R.ORDER_RCM, R.ORDER_GIVEN):
        grid = R.Grid(ctx, xyz, st, order=order)
        der = R.RBFFD(R.LSFC, grid, 2)
        der.setWeights(R.LSFC, W)
        assert np.array_equal(der.getWeights(R.LSFC), W)
        pde = R.HeatSphere(grid, der, 1.0, dtype=R.F64)
        pde.setShape(1, 128)
        pde.fillInitialConditions(u0)
        pde.advance(R.RK4, 1e-5, 12)
        outs[order] = pde.getLocalSolution()
        pde.close()
        grid.close()
    ctx.close()
    for order, out in outs.items():
        assert np.array_equal(out, ref), order
