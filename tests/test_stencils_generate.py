"""Grid::generateStencils with the reference's default brute-force generator
and its k-d tree, max_st_radius trimming included
(src/grids/grid_interface.cpp:514-536, 637-725), against the reference's own
code compiled from its sources into oracle/_ref/libref_grid.so (a C wrapper
in oracle/ref_grid.cpp).  Host only."""
import numpy as np
import pytest

import oracle as O
import rbffd_gpu_b200 as R

needs_ref = pytest.mark.skipif(O.ref_lib("ref_grid") is None, reason="reference sources not built")


def _compare(xyz, n, method, max_radius=1.7976931348623157e308):
    st, ln = R.generate_stencils(xyz, n, method, max_radius)
    ref_st, ref_ln = O.ref_stencils_generate(xyz, n, method, max_radius)
    assert np.array_equal(ln, ref_ln)
    for i in range(len(xyz)):
        assert np.array_equal(st[i, :ln[i]], ref_st[i, :ln[i]]), i
        assert (st[i, ln[i]:] == i).all()  # padding: the centre
    return st, ln


@needs_ref
@pytest.mark.parametrize("method", [R.ST_BRUTE_FORCE, R.ST_KDTREE])
@pytest.mark.parametrize("N,n,seed", [(800, 17, 1), (1500, 31, 2), (600, 50, 3)])
def test_sphere_nodes(method, N, n, seed):
    xyz = R.fibonacci_nodes(N, seed)
    st, ln = _compare(xyz, n, method)
    assert (ln == n).all() and (st[:, 0] == np.arange(N)).all()


@needs_ref
@pytest.mark.parametrize("method", [R.ST_BRUTE_FORCE, R.ST_KDTREE])
def test_radius_trimming(method):
    xyz = R.fibonacci_nodes(1000, 5)
    for r in (0.05, 0.12, 0.2):
        st, ln = _compare(xyz, 31, method, r)
        assert ln.min() >= 1 and ln.max() <= 31
    assert ln.min() < 31  # the largest radius still trims some stencils


@needs_ref
def test_brute_force_ties_in_decreasing_index():
    """A cubic lattice: every node has many neighbours at equal distance. The
    brute-force generator keeps the higher node numbers first among equal
    distances (its std::set with a `<=` comparator) and equals the reference
    entry for entry.  The k-d tree's order among exact ties follows its
    search; the product orders them by index, so there the distance lists
    agree, not the tied members."""
    g = np.arange(7, dtype=np.float64)
    xyz = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) * 0.1
    bf, _ = _compare(xyz, 19, R.ST_BRUTE_FORCE)
    kd, _ = R.generate_stencils(xyz, 19, R.ST_KDTREE)
    ref_kd, _ = O.ref_stencils_generate(xyz, 19, R.ST_KDTREE)
    dist = lambda st: ((xyz[st] - xyz[:, None, :]) ** 2).sum(2)
    assert np.array_equal(dist(kd), dist(ref_kd))
    assert not np.array_equal(bf, kd)
    centre = 3 * 49 + 3 * 7 + 3
    d = ((xyz[bf[centre]] - xyz[centre]) ** 2).sum(1)
    for a in range(1, 19):
        if d[a] == d[a - 1]:
            assert bf[centre, a] < bf[centre, a - 1]


def test_invalid_radius():
    with pytest.raises(R.RbffdError):
        R.generate_stencils(R.fibonacci_nodes(100, 1), 9, R.ST_BRUTE_FORCE, 0.0)


@needs_ref
def test_duplicate_point_order():
    """A duplicated node: the brute-force generator puts the copy with the
    higher number first, ahead of the centre, as the reference does; the k-d
    tree lists keep the centre first."""
    xyz = R.fibonacci_nodes(300, 7)
    xyz = np.vstack([xyz, xyz[5:6]])
    bf, _ = _compare(xyz, 12, R.ST_BRUTE_FORCE)
    assert bf[5, 0] == 300 and bf[5, 1] == 5
    kd, _ = R.generate_stencils(xyz, 12, R.ST_KDTREE)
    assert kd[5, 0] == 5 and kd[300, 0] == 300


def test_variable_epsilon_equals_oracle():
    """RBFFD::setVariableEpsilon (Sarler 2006 form) on ragged stencils:
    1 / (alpha * distance to the last node), bit for bit with the oracle."""
    xyz = R.fibonacci_nodes(1200, 4)
    st, ln = R.generate_stencils(xyz, 31, R.ST_KDTREE, 0.11)
    for alpha in (1.0, 0.37):
        got = R.variable_epsilon(xyz, st, ln, alpha)
        assert np.array_equal(got, O.variable_epsilon(xyz, st, ln, alpha, np.ones(len(xyz))))
    full = R.knn_stencils(xyz, 17)
    assert np.array_equal(R.variable_epsilon(xyz, full, None, 2.0),
                          O.variable_epsilon(xyz, full, None, 2.0, np.ones(len(xyz))))
    with pytest.raises(R.RbffdError):
        R.variable_epsilon(xyz, st, ln, 0.0)


def test_generator_argument_checks():
    """Invalid calls return RBFFD_ERR_INVALID (the C ABI never exits)."""
    from rbffd_gpu_b200 import _lib
    L = _lib.load()
    xyz = R.fibonacci_nodes(50, 1)
    st = np.zeros((50, 5), dtype=np.int32)
    ln = np.zeros(50, dtype=np.int32)
    dp = xyz.ctypes.data_as(_lib.dp)
    ip, lp = st.ctypes.data_as(_lib.ip), ln.ctypes.data_as(_lib.ip)
    assert L.rbffd_stencils_generate(dp, 50, 5, 7, 1.0, ip, lp, None, 0) == -1      # unknown method
    assert L.rbffd_stencils_generate(dp, 50, 5, 0, -1.0, ip, lp, None, 0) == -1     # radius <= 0
    assert L.rbffd_stencils_generate(dp, 50, 51, 0, 1.0, ip, lp, None, 0) == -1     # n > N
    assert L.rbffd_stencils_generate(None, 50, 5, 0, 1.0, ip, lp, None, 0) == -1    # no nodes
    assert L.rbffd_stencils_generate(dp, 50, 5, 0, 1.0, ip, None, None, 0) == 0     # lengths optional
    bad = np.full((50, 5), 60, dtype=np.int32)
    eps = np.ones(50)
    assert L.rbffd_variable_epsilon(50, dp, 5, bad.ctypes.data_as(_lib.ip), None, 1.0,
                                    eps.ctypes.data_as(_lib.dp)) == -1              # index out of range
