"""Pins against committed outputs of the reference's own code
(tests/golden/reference_outputs.npz, written by tests/golden/make_golden.py
from the reference sources compiled into oracle/_ref/).  These run without
the reference tree: the oracle's RBF and cart2sph restatements and the
product's host stencil generators and norms must reproduce the reference's
outputs bit for bit."""
import os

import numpy as np
import pytest

import oracle as O
import rbffd_gpu_b200 as R

GOLDEN = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_outputs.npz"))


def test_oracle_rbf_gaussian_equals_reference_outputs():
    """RBF_Gaussian (src/rbffd/rbfs/rbf_gaussian.h): eval, derivatives,
    Laplacians, hyperviscosity."""
    for (which, eps, dim, dx, dy, dz, k), ref in zip(GOLDEN["rbf_args"], GOLDEN["rbf_vals"]):
        got = O.lib().orc_rbf(int(which), eps, int(dim), dx, dy, dz, int(k))
        assert got == ref or (np.isnan(got) and np.isnan(ref)), (which, eps, dim, k, got, ref)


def test_oracle_cart2sph_equals_reference_outputs():
    for p, ref in zip(GOLDEN["sph_xyz"], GOLDEN["sph_vals"]):
        assert O.cart2sph(*p) == tuple(ref)


def test_knn_equals_reference_kdtree_outputs():
    assert np.array_equal(R.knn_stencils(GOLDEN["kd_xyz"], 17), GOLDEN["kd_st"])


def test_brute_force_with_radius_equals_reference_outputs():
    st, ln = R.generate_stencils(GOLDEN["bf_xyz"], 15, R.ST_BRUTE_FORCE, 0.2)
    assert np.array_equal(ln, GOLDEN["bf_len"])
    for i in range(len(ln)):
        assert np.array_equal(st[i, :ln[i]], GOLDEN["bf_st"][i, :ln[i]])


def test_hash_stencils_equal_reference_outputs():
    order, st, ln = R.stencils_hash(GOLDEN["hash_xyz"], 20, (8, 12, 6))
    assert np.array_equal(order, GOLDEN["hash_order"])
    assert np.array_equal(ln, GOLDEN["hash_len"])
    for i in range(len(ln)):
        assert np.array_equal(st[i, :ln[i]], GOLDEN["hash_st"][i, :ln[i]])


@pytest.mark.parametrize("row", range(4))
def test_sol_norms_equal_reference_outputs(row):
    got = R.sol_norms(GOLDEN["norms_sol"][row], GOLDEN["norms_exact"][row])
    keys = ("l1", "l1_rel", "l2", "l2_rel", "linf", "linf_rel")
    assert np.array_equal(np.array([got[k] for k in keys]), GOLDEN["norms_vals"][row])


def test_oracle_core_equals_reference_outputs():
    """The reference's RBFFD weights, applyWeightsForDeriv and CosineBell RK4
    (src/rbffd/rbffd.cpp, src/pdes/time_dependent_pde.cpp,
    src/pdes/hyperbolic/cosine_bell.cpp, compiled from its sources) on 300
    nodes: the oracle with the constant basis and the reference's arithmetic
    (oracle.reference_arithmetic) reproduces them bit for bit."""
    xyz, st = GOLDEN["core_xyz"], GOLDEN["core_st"]
    N, n = st.shape
    assert np.array_equal(R.knn_stencils(xyz, n), st)
    W = O.weights(xyz, st, None, 0.4 / np.sqrt(4 * np.pi / N), O.LAMBDA | O.THETA | O.HV, dim=2, poly_deg=0,
                  hv_k=4, hv_scale=-1e-3 * float(N) ** -4.0)
    u = np.sin(3 * xyz[:, 0]) + xyz[:, 1] * xyz[:, 2]
    with O.reference_arithmetic():
        for name, t in (("lambda", O.LAMBDA), ("theta", O.THETA), ("hv", O.HV)):
            assert np.array_equal(W[t], GOLDEN["core_w_" + name][:, :n]), name
            assert np.array_equal(O.apply(st, None, W[t], u), GOLDEN["core_apply_" + name]), name
        h0 = GOLDEN["core_h0"]
        assert np.array_equal(R.exact_cosine_bell(xyz), h0)
        cu, cv = O.cosine_bell_coeffs(xyz, 1.0, np.pi / 2, 2 * np.pi / 1036800.0)
        for k in (1, 5):
            got = O.rk4_advect(st, None, W[O.LAMBDA], W[O.THETA], W[O.HV], cu, cv, h0, 1036.8, k)
            assert np.array_equal(got, GOLDEN["core_rk4_%d" % k]), k
