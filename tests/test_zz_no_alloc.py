"""The allocation-free heat RK4 entry point, rbffd_heat_rk4_noalloc.

It is for callers that cannot let the library allocate device memory (an
application that has reserved the GPU's memory for its own pool, or a loop
where a cudaMalloc/cudaFree would synchronise the device).  It keeps the RK4
stage buffers in a fixed array inside the library, so these tests check that
it gives the same states as the regular PDE entry point (rbffd_pde_advance,
one lane per stencil row: the same arithmetic, so the results must be
identical) on two calls in a row -- the second call starts from what the
first left in that shared array -- that it allocates nothing, and that grids
larger than its fixed array are refused.

This file is named so that pytest collects it last.
"""
import ctypes
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as O
import rbffd_gpu_b200 as R
from tests.helpers import sphere_problem

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def heat_grid(ctx):
    N, n = 4096, 31
    xyz, st = sphere_problem(N, n, 1)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(R.LSFC, grid, 2)
    der.setEpsilon(0.25 / np.sqrt(4 * np.pi / N))
    der.setPolynomialDegree(2)
    der.computeAllWeightsForAllStencils()
    lmax = 10
    u0 = R.exact_sph_heat(xyz, lmax, np.random.default_rng(7).standard_normal((lmax + 1) ** 2), 0.0)
    yield grid, der, u0
    grid.close()


def _reference_states(grid, der, u0, dtype, dt, steps):
    pde = R.HeatSphere(grid, der, 1.0, dtype=dtype)
    pde.setShape(1, 256)
    pde.fillInitialConditions(u0)
    out = []
    for k in steps:
        pde.advance(R.RK4, dt, k)
        out.append(pde.getLocalSolution())
    pde.close()
    return out


@pytest.mark.parametrize("dtype", [R.F64, R.F32])
def test_noalloc_matches_pde_entry_point_on_two_calls(ctx, heat_grid, dtype):
    grid, der, u0 = heat_grid
    dt = 2e-5
    ref1, ref2 = _reference_states(grid, der, u0, dtype, dt, (7, 5))
    tdt = torch.float64 if dtype == R.F64 else torch.float32
    u = torch.tensor(u0, dtype=tdt, device="cuda")
    torch.cuda.synchronize()
    held0, free0, _ = ctx.mem_info()
    torch_alloc0 = torch.cuda.memory_allocated()
    L = ctx.L
    ctx.check(L.rbffd_heat_rk4_noalloc(grid.h, dtype, 1.0, dt, 7, ctypes.c_void_p(u.data_ptr())), "noalloc call 1")
    got1 = u.double().cpu().numpy()
    ctx.check(L.rbffd_heat_rk4_noalloc(grid.h, dtype, 1.0, dt, 5, ctypes.c_void_p(u.data_ptr())), "noalloc call 2")
    got2 = u.double().cpu().numpy()
    held1, free1, _ = ctx.mem_info()
    assert held1 == held0
    assert torch.cuda.memory_allocated() == torch_alloc0
    # same kernel and arithmetic as the PDE entry point with one lane per row: identical states
    assert np.array_equal(got1, ref1)
    assert np.array_equal(got2, ref2)


def test_noalloc_fp64_matches_oracle(ctx, heat_grid):
    grid, der, u0 = heat_grid
    W = der.getWeights(R.LSFC)
    u = torch.tensor(u0, dtype=torch.float64, device="cuda")
    ctx.check(ctx.L.rbffd_heat_rk4_noalloc(grid.h, R.F64, 1.0, 2e-5, 6, ctypes.c_void_p(u.data_ptr())), "noalloc")
    ref = O.rk4_heat(grid.stencils, None, W, u0, 2e-5, 6)
    assert np.array_equal(u.cpu().numpy(), ref)


def test_noalloc_rejects_grids_beyond_its_fixed_scratch(ctx):
    N, n = 262145, 7  # one node more than the FP64 limit
    xyz = R.fibonacci_nodes(N, 11)
    st = R.knn_stencils(xyz, n)
    grid = R.Grid(ctx, xyz, st)
    u = torch.zeros(N, dtype=torch.float64, device="cuda")
    rc = ctx.L.rbffd_heat_rk4_noalloc(grid.h, R.F64, 1.0, 1e-6, 1, ctypes.c_void_p(u.data_ptr()))
    assert rc == -1
    assert b"at most 262144" in ctx.L.rbffd_ctx_last_error(ctx.h)
    grid.close()


_FRESH = r"""
import ctypes, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import torch
import rbffd_gpu_b200 as R

ctx = R.Context(0)  # loads the allocation-free path's device code on this GPU


def heat_grid(N, seed):
    xyz = R.fibonacci_nodes(N, seed)
    grid = R.Grid(ctx, xyz, R.knn_stencils(xyz, 31))
    der = R.RBFFD(R.LSFC, grid, 2)
    der.setEpsilon(0.25 / np.sqrt(4 * np.pi / N))
    der.setPolynomialDegree(2)
    der.computeAllWeightsForAllStencils()
    u = torch.tensor(R.exact_sph_heat(xyz, 4, np.ones(25), 0.0), dtype=torch.float64, device="cuda")
    return grid, der, u


def call(grid, u):
    ctx.check(ctx.L.rbffd_heat_rk4_noalloc(grid.h, R.F64, 1.0, 1e-5, 3, ctypes.c_void_p(u.data_ptr())), "noalloc")


free = []
g1, d1, u1 = heat_grid(4096, 1)
torch.cuda.synchronize()
free.append(ctx.mem_info()[1])
call(g1, u1)  # the first call on this device in this process
free.append(ctx.mem_info()[1])
g2, d2, u2 = heat_grid(10242, 3)  # a new grid, allocated before the next reading
torch.cuda.synchronize()
free.append(ctx.mem_info()[1])
call(g2, u2)
free.append(ctx.mem_info()[1])
print(json.dumps(free))
"""


def test_noalloc_takes_no_device_memory_in_a_fresh_process():
    """In a process of its own (nothing else has run): once the context
    exists, neither the first call of the entry point nor a later call on a
    new grid changes the GPU's free memory (cudaMemGetInfo) -- no allocation,
    and no module loaded by the call."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _FRESH, root], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    f0, f1, f2, f3 = json.loads(r.stdout.strip().splitlines()[-1])
    assert f1 == f0, "first call changed free device memory by %d bytes" % (f0 - f1)
    assert f3 == f2, "second call changed free device memory by %d bytes" % (f2 - f3)
