"""The two arms of the benchmark measure the same workload: the CPU arm
(bench.py --impl reference) builds its grid and initial state from the
oracle and the reference's own k-d tree, never from the product library, and
both arms print the same config dict."""
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402
import oracle as O  # noqa: E402
import rbffd_gpu_b200 as R  # noqa: E402


def test_oracle_nodes_equal_the_product_nodes():
    for N, seed in ((1000, 77), (4096, 1), (40962, 2)):
        assert np.array_equal(O.fibonacci_nodes(N, seed), R.fibonacci_nodes(N, seed))


def test_oracle_harmonic_sum_equals_the_product_initial_state():
    xyz = R.fibonacci_nodes(10242, 2)
    c = np.random.default_rng(2).standard_normal(21 * 21)
    for t in (0.0, 5e-4):
        a, b = O.sph_heat(xyz, 20, c, t), R.exact_sph_heat(xyz, 20, c, t)
        assert np.abs(a - b).max() <= 1e-14 * np.abs(b).max()


def test_reference_arm_setup_does_not_load_the_product():
    """The CPU arm's set-up at the benchmark's full size (N = 163842, n = 50),
    in a fresh interpreter: the stencils equal the product's lists and no
    product library is mapped into the process."""
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r)\n"
        "import bench\n"
        "xyz, st, u0, eps, c, src = bench.setup_problem_reference()\n"
        "np.save(sys.argv[1], st)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('PRODUCT' if 'librbffd_sm100' in maps or 'rbffd_gpu_b200' in sys.modules else 'CLEAN', src)\n" % ROOT)
    out = os.path.join(ROOT, "tests", ".bench_arm_st.npy")
    try:
        r = subprocess.run([sys.executable, "-c", code, out], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        assert r.stdout.startswith("CLEAN"), r.stdout
        st = np.load(out)
    finally:
        if os.path.exists(out):
            os.remove(out)
    W = bench.WORKLOAD
    xyz = R.fibonacci_nodes(W["N"], W["seed"])
    assert np.array_equal(st, R.knn_stencils(xyz, W["n"]))


def test_both_arms_print_one_config():
    assert bench.workload_config(1) == bench.workload_config(1)
    cfg = bench.workload_config(1)
    assert cfg["nodes"] == 163842 and cfg["stencil"] == 50 and cfg["rk4_steps"] == 500
    src = open(os.path.join(ROOT, "bench.py")).read()
    # each arm's JSON line takes its config from workload_config and nowhere else
    assert src.count('"config": workload_config(ws)') == 2
