"""Writes tests/golden/reference_outputs.npz: outputs of the reference's own
code, compiled from its sources into oracle/_ref/ (oracle/build.py), on small
seeded inputs.  The tests in tests/test_golden.py check the oracle and the
product's host functions against these arrays without needing the reference
tree.  Run from the repository root where the reference tree is present:

    python tests/golden/make_golden.py

Contents (all from the reference's code):
  rbf_*      RBF_Gaussian eval/derivatives/Laplacians/hyperviscosity
             (src/rbffd/rbfs/rbf_gaussian.h) at seeded (which, eps, dim, d, k)
  sph_*      cart2sph (src/utils/geom/cart2sph.cpp) of 200 Fibonacci nodes
  kd_*       KDTree::k_closest_points lists (external/kdtree/KDTree.h), 600 nodes, n = 17
  bf_*       Grid::generateStencilsBruteForce, 400 nodes, n = 15, with max_st_radius 0.2
  hash_*     Grid::generateStencilsHash, 600 nodes, n = 20, 8x12x6 overlay (order, stencils, lengths)
  norms_*    norms.cpp l1/l2/linf with calcSolNorms' relative rule on seeded vectors
  core_*     the reference's RBFFD + CosineBell + TimeDependentPDE (oracle/ref_rbffd.cpp):
             300 nodes, n = 13, eps = 0.4 / h, LAMBDA, THETA, HV (k = 4, gamma = 1e-3, dim 2):
             k-d tree stencils, the stored weights (n + 1 per row), applyWeightsForDeriv of a
             smooth field per operator, and the cosine bell after 1 and 5 RK4 steps of 1036.8 s
"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle as O  # noqa: E402
import rbffd_gpu_b200 as R  # noqa: E402


def main():
    L = O.ref_lib("ref_rbf")
    if L is None or O.ref_lib("ref_kdtree") is None or O.ref_lib("ref_grid") is None or \
            O.ref_lib("ref_norms") is None or not O.RefRBFFD.available():
        sys.exit("the reference libraries are not built (python -c 'import oracle.build as b; b.build()')")
    out = {}
    rng = np.random.default_rng(2024)
    args, vals = [], []
    for which in range(9):
        for _ in range(40):
            d = rng.normal(size=3) * rng.choice([1e-3, 1e-1, 0.5])
            eps = rng.uniform(0.5, 9.0)
            dim = int(rng.integers(1, 4))
            k = int(rng.integers(0, 9))
            args.append([which, eps, dim, d[0], d[1], d[2], k])
            vals.append(L.ref_rbf(which, eps, dim, *d, k))
    out["rbf_args"] = np.array(args)
    out["rbf_vals"] = np.array(vals)
    xyz = R.fibonacci_nodes(200, 11)
    sph = []
    for p in xyz:
        t, ph, r = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        L.ref_cart2sph(*p, ctypes.byref(t), ctypes.byref(ph), ctypes.byref(r))
        sph.append([t.value, ph.value])
    out["sph_xyz"], out["sph_vals"] = xyz, np.array(sph)
    xyz = R.fibonacci_nodes(600, 12)
    out["kd_xyz"], out["kd_st"] = xyz, O.ref_knn(xyz, 17)[0]
    xyz = R.fibonacci_nodes(400, 13)
    st, ln = O.ref_stencils_generate(xyz, 15, 0, 0.2)
    out["bf_xyz"], out["bf_st"], out["bf_len"] = xyz, st, ln
    xyz = R.fibonacci_nodes(600, 14)
    order, st, ln = O.ref_stencils_hash(xyz, 20, (8, 12, 6))
    out["hash_xyz"], out["hash_order"], out["hash_st"], out["hash_len"] = xyz, order, st, ln
    sol = rng.normal(size=(4, 300))
    exact = sol + 1e-3 * rng.normal(size=(4, 300))
    exact[3] = 0.0  # the calcSolNorms rule for exact norms below 1e-10
    out["norms_sol"], out["norms_exact"] = sol, exact
    out["norms_vals"] = np.array([O.ref_sol_norms(sol[i], exact[i]) for i in range(4)])
    N, n = 300, 13
    xyz = R.fibonacci_nodes(N, 21)
    ref = O.RefRBFFD(xyz, n, O.LAMBDA | O.THETA, 0.4 / np.sqrt(4 * np.pi / N), dim=2, hv_k=4, hv_gamma=1e-3,
                     use_hv=True)
    out["core_xyz"], out["core_st"] = xyz, ref.stencils
    u = np.sin(3 * xyz[:, 0]) + xyz[:, 1] * xyz[:, 2]
    for name, t in (("lambda", O.LAMBDA), ("theta", O.THETA), ("hv", O.HV)):
        out["core_w_" + name] = ref.weights(t)
        out["core_apply_" + name] = ref.apply(t, u)
    h0 = R.exact_cosine_bell(xyz)
    out["core_h0"] = h0
    out["core_rk4_1"] = ref.rk4(O.RefRBFFD.KIND_COSINE_BELL, h0, 1036.8, 1)
    out["core_rk4_5"] = ref.rk4(O.RefRBFFD.KIND_COSINE_BELL, h0, 1036.8, 5)
    ref.close()
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_outputs.npz"), **out)


if __name__ == "__main__":
    main()
