"""The C ABI library: it loads, exports every function include/rbffd_sm100.h
declares, and its host-side entry points work without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import rbffd_gpu_b200 as R
from rbffd_gpu_b200 import _lib
from tests.helpers import has_gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for f in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(rbffd_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # the Python binding covers the same set
    assert set(names) <= set(_lib.PROTOTYPES), set(names) - set(_lib.PROTOTYPES)


def test_exported_symbols_are_c_linkage():
    out = os.popen("nm -D --defined-only %s" % _lib.LIB_PATH).read()
    for n in declared_functions():
        assert re.search(r"\bT %s$" % n, out, re.M), n


def test_version_and_status_strings():
    assert "sm_100a" in R.version()
    L = _lib.load()
    for s in range(0, -10, -1):
        assert L.rbffd_status_string(s)
    assert L.rbffd_status_string(-9).decode() == "no CUDA device"


def test_context_without_device_reports_no_device():
    if has_gpu():
        pytest.skip("a GPU is present")
    L = _lib.load()
    h = ctypes.c_void_p()
    assert L.rbffd_ctx_create(0, ctypes.byref(h)) == -9
    assert R.device_count() == 0


def test_null_handles_are_rejected():
    L = _lib.load()
    assert L.rbffd_ctx_destroy(None) == -1
    assert L.rbffd_grid_destroy(None) == -1
    assert L.rbffd_pde_destroy(None) == -1
    assert L.rbffd_pde_advance(None, 2, 1.0, 1, 0) == -1
    assert L.rbffd_apply(None, 1, 1, 0, 1, None, None) == -1
    assert L.rbffd_pde_set_compensated_state(None, 1) == -1


def test_fibonacci_nodes_are_unit_and_seeded():
    a = R.fibonacci_nodes(1000, 3)
    b = R.fibonacci_nodes(1000, 3)
    c = R.fibonacci_nodes(1000, 4)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert np.abs(np.linalg.norm(a, axis=1) - 1).max() < 4e-16


def test_knn_centre_first_and_sorted():
    xyz = R.fibonacci_nodes(2000, 9)
    st = R.knn_stencils(xyz, 17)
    assert (st[:, 0] == np.arange(2000)).all()
    d = np.linalg.norm(xyz[st] - xyz[:, None, :], axis=2)
    assert (np.diff(d, axis=1) >= 0).all()
    # brute force agreement on a subset
    for i in range(0, 2000, 97):
        dd = ((xyz - xyz[i]) ** 2).sum(1)
        assert set(np.argsort(dd, kind="stable")[:17]) == set(st[i])


def test_knn_rejects_bad_sizes():
    xyz = R.fibonacci_nodes(10, 1)
    with pytest.raises(R.RbffdError):
        R.knn_stencils(xyz, 11)


def test_sph_heat_exact_is_eigenfunction_decay():
    xyz = R.fibonacci_nodes(500, 2)
    lmax = 4
    c = np.zeros((lmax + 1) ** 2)
    c[3 * 3 + 3] = 1.0  # l = 3, m = 0
    u0 = R.exact_sph_heat(xyz, lmax, c, 0.0)
    u1 = R.exact_sph_heat(xyz, lmax, c, 0.1)
    assert np.allclose(u1, u0 * np.exp(-12 * 0.1), rtol=1e-13, atol=1e-15)
    # orthonormal: mean of Y^2 over the sphere ~ 1/(4 pi)
    assert abs(np.mean(u0 ** 2) * 4 * np.pi - 1) < 0.05


def test_cosine_bell_exact_solution_shape():
    xyz = R.fibonacci_nodes(4096, 1)
    h = R.exact_cosine_bell(xyz)
    assert h.max() <= 1.0 and h.min() == 0.0
    assert 0.02 < (h > 0).mean() < 0.04  # cap of radius 1/3 covers (1-cos(1/3))/2 of the sphere


def test_server_rejects_null_handles():
    L = _lib.load()
    assert L.rbffd_server_start(None, 0.8, 0, None) == -1
    assert L.rbffd_server_submit(None, None, None) == -1
    assert L.rbffd_server_stop(None) == -1
    assert L.rbffd_server_cancel(None, 1) == -1
    assert L.rbffd_server_wait_idle(None, 1.0) == -1
    assert L.rbffd_server_set_admission_order(None, 1) == -1
    with pytest.raises(ValueError):
        R.Server(None, admission="longest")  # checked before any call into the library


def test_ctypes_structs_match_the_header_layout(tmp_path):
    """The Python binding's structs have the C compiler's sizes and offsets."""
    structs = {"rbffd_pde_params": _lib.PdeParams, "rbffd_request": _lib.Request,
               "rbffd_server_stats": _lib.ServerStats, "rbffd_weight_params": _lib.WeightParams,
               "rbffd_eig_output": _lib.EigOutput}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "rbffd_sm100.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (cname, cname))
        for f, _ in py._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, f, cname, f))
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    assert os.system("gcc -std=c99 -I%s %s -o %s" % (os.path.join(ROOT, "include"), src, exe)) == 0
    got = {}
    for line in os.popen(str(exe)).read().splitlines():
        a, b, c = line.split()
        got[(a, b)] = int(c)
    for cname, py in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)
