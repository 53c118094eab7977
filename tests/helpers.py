"""Shared problem set-ups for the tests (seeded, deterministic)."""
import glob
import os

import numpy as np

import rbffd_gpu_b200 as R

_CACHE = {}


def sphere_problem(N, n, seed):
    """Fibonacci nodes (seeded rotation) and their n-nearest-neighbour stencils."""
    key = (N, n, seed)
    if key not in _CACHE:
        xyz = R.fibonacci_nodes(N, seed)
        st = R.knn_stencils(xyz, n)
        _CACHE[key] = (xyz, st)
    return _CACHE[key]


def cosine_bell_setup(N=4096, n=31):
    """Cosine-bell parameters in the reference's units: sphere radius 1, one
    revolution = 1036800 s in 1000 steps (tests/experiments/cosine_bell_on_sphere/test.conf)."""
    T = 1036800.0
    return dict(a=1.0, alpha=np.pi / 2, T=T, u0=2 * np.pi / T, dt=T / 1000.0)


def sph_coeffs(lmax, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((lmax + 1) ** 2)


def rel_l2(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def rel_linf(a, b):
    return float(np.abs(np.ravel(a) - np.ravel(b)).max() / np.abs(np.ravel(b)).max())


def has_gpu():
    """A CUDA device node is present (the same test as conftest's)."""
    return os.path.exists("/dev/nvidiactl") or bool(glob.glob("/dev/nvidia[0-9]*"))
