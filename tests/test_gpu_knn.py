"""GPU stencil search (rbffd_stencils_knn_gpu) against the host search, which
the oracle pins bit-exactly to the reference k-d tree
(external/kdtree/KDTree.h:407-433): identical ordered lists and tie counts."""
import numpy as np
import pytest

import rbffd_gpu_b200 as R

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,n,seed", [(20000, 17, 3), (20000, 31, 1), (40962, 50, 2), (30000, 101, 4)])
def test_knn_gpu_equals_host_on_sphere(ctx, N, n, seed):
    xyz = R.fibonacci_nodes(N, seed)
    host, th = R.knn_stencils(xyz, n, return_ties=True)
    dev, td = R.knn_stencils_gpu(ctx, xyz, n, return_ties=True)
    assert np.array_equal(dev, host)
    assert td == th
    assert (dev[:, 0] == np.arange(N)).all()


def test_knn_gpu_ties_on_a_lattice(ctx):
    """A cubic lattice: most distance lists have exact ties, broken by index."""
    g = np.arange(12, dtype=np.float64)
    xyz = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) * 0.1
    host, th = R.knn_stencils(xyz, 27, return_ties=True)
    dev, td = R.knn_stencils_gpu(ctx, xyz, 27, return_ties=True)
    assert th > 1000 and td == th
    assert np.array_equal(dev, host)


def test_knn_gpu_duplicates_and_all_points(ctx):
    rng = np.random.default_rng(7)
    xyz = rng.normal(size=(500, 3))
    xyz[250:260] = xyz[100:110]  # duplicated points: distance 0 ahead of the centre
    for n in (9, 64, 255):
        assert np.array_equal(R.knn_stencils_gpu(ctx, xyz, n), R.knn_stencils(xyz, n))
    small = xyz[:40]
    assert np.array_equal(R.knn_stencils_gpu(ctx, small, 40), R.knn_stencils(small, 40))


def test_knn_gpu_rejects_bad_sizes(ctx):
    xyz = R.fibonacci_nodes(300, 1)
    with pytest.raises(R.RbffdError):
        R.knn_stencils_gpu(ctx, xyz, 256)
    with pytest.raises(R.RbffdError):
        R.knn_stencils_gpu(ctx, xyz, 301)


@pytest.mark.parametrize("method", [R.ST_BRUTE_FORCE, R.ST_KDTREE])
@pytest.mark.parametrize("max_radius", [1.7976931348623157e308, 0.06])
def test_generators_on_device_equal_host(ctx, method, max_radius):
    """Both reference generators (brute-force order, k-d tree) with and without
    the stencil radius: device lists and lengths equal the host's."""
    xyz = R.fibonacci_nodes(20000, 9)
    st, ln = R.generate_stencils_gpu(ctx, xyz, 31, method, max_radius)
    hs, hl = R.generate_stencils(xyz, 31, method, max_radius)
    assert np.array_equal(ln, hl) and np.array_equal(st, hs)
    if max_radius < 1.0:
        assert ln.min() < 31


def test_brute_force_ties_on_device(ctx):
    g = np.arange(8, dtype=np.float64)
    xyz = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) * 0.1
    xyz = np.vstack([xyz, xyz[100:101]])  # and a duplicated point
    for method in (R.ST_BRUTE_FORCE, R.ST_KDTREE):
        st, ln = R.generate_stencils_gpu(ctx, xyz, 27, method)
        hs, hl = R.generate_stencils(xyz, 27, method)
        assert np.array_equal(st, hs) and np.array_equal(ln, hl)
