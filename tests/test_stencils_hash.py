"""Hash-grid stencils (Grid::generateStencilsHash, src/grids/grid_interface.cpp:733-966,
the generator of the reference's cosine-bell experiment) against the
reference's own code, compiled from its sources into oracle/_ref: the same
node renumbering, stencil lengths and stencils, entry for entry, for several
overlay shapes (including y and z cell counts that differ, where the
reference bounds the z index by the y count), radius trimming, given
extents, and a lattice full of equal distances (the tie order)."""
import numpy as np
import pytest

import oracle as O
import rbffd_gpu_b200 as R

pytestmark = pytest.mark.skipif(O.ref_lib("ref_grid") is None, reason="reference sources not built")


def _compare(xyz, n, dims=(10, 10, 10), extents=None, max_radius=1.7976931348623157e308):
    o, st, ln = R.stencils_hash(xyz, n, dims, extents, max_radius)
    ro, rst, rln = O.ref_stencils_hash(xyz, n, dims, extents, max_radius)
    assert np.array_equal(o, ro)
    assert np.array_equal(ln, rln)
    mask = np.arange(n)[None, :] < ln[:, None]
    assert np.array_equal(np.where(mask, st, -1), rst)
    centre_first = st[:, 0] == np.arange(len(xyz))
    if dims[2] <= dims[1]:
        assert np.all(centre_first)
    else:  # z cells at or past the y count are skipped: some nodes miss their own cell
        assert not np.all(centre_first)
    return o, st, ln


@pytest.mark.parametrize("N,n,dims,seed", [(2562, 31, (10, 10, 10), 1), (4096, 50, (8, 12, 6), 2),
                                           (3000, 17, (10, 6, 14), 3), (642, 9, (4, 4, 4), 4),
                                           (1000, 101, (10, 10, 10), 5)])
def test_equals_reference(N, n, dims, seed):
    _compare(R.fibonacci_nodes(N, seed), n, dims)


def test_radius_trims_stencils():
    o, st, ln = _compare(R.fibonacci_nodes(2562, 1), 31, max_radius=0.12)
    assert ln.min() < 31 and ln.max() <= 31


def test_given_extents():
    _compare(R.fibonacci_nodes(2000, 6), 21, (6, 6, 6), extents=[-1.2, 1.2, -1.1, 1.3, -1.0, 1.0])


def test_ties_on_a_lattice():
    g = np.arange(9, dtype=np.float64) * 0.125
    xyz = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    _compare(xyz, 27, (4, 4, 4))


def test_not_an_exact_knn():
    """Candidates come from nearby cells only: some stencils differ from the
    exact nearest neighbours (which rbffd_stencils_knn computes)."""
    xyz = R.fibonacci_nodes(2562, 1)
    o, st, _ = R.stencils_hash(xyz, 31)
    exact = R.knn_stencils(xyz[o], 31)
    differ = np.mean([set(a) != set(b) for a, b in zip(st, exact)])
    assert 0.0 < differ < 0.1


def test_rejects_what_the_reference_cannot_finish():
    xyz = R.fibonacci_nodes(100, 1)
    with pytest.raises(R.RbffdError):
        R.stencils_hash(xyz, 101)  # more stencil nodes than nodes
    with pytest.raises(R.RbffdError):
        R.stencils_hash(xyz, 10, extents=[0, 0.5, 0, 0.5, 0, 0.5])  # nodes outside the extents
    with pytest.raises(R.RbffdError):
        R.stencils_hash(xyz, 10, (0, 10, 10))
