"""Weight files in the reference's Matrix Market forms (RBFFD::writeToAsciiFile /
writeToBinaryFile, src/rbffd/rbffd.cpp:1265-1375; loadFromAsciiFile /
loadFromBinaryFile, rbffd.cpp:983-1210): exact round trips, the header as
the reference's own NIST routines (external/nist/mmio.cpp) write and read it,
the reference's entry forms, and refusal of files for other stencils."""
import ctypes
import os

import numpy as np
import pytest

import oracle as O
import rbffd_gpu_b200 as R


def _case(N=300, n_pad=12, seed=0):
    rng = np.random.default_rng(seed)
    lens = rng.integers(3, n_pad + 1, N).astype(np.int32)
    st = np.zeros((N, n_pad), dtype=np.int32)
    w = np.zeros((N, n_pad))
    for i in range(N):
        others = rng.choice(np.delete(np.arange(N), i), n_pad - 1, replace=False)
        st[i] = np.concatenate([[i], others])
        w[i, :lens[i]] = rng.standard_normal(lens[i]) * 10.0 ** rng.integers(-8, 8, lens[i])
    return st, lens, w


def _ref_mmio():
    L = O.ref_lib("ref_mmio")
    if L is None:
        pytest.skip("reference mmio not built here")
    return L


def _ref_header(L, path):
    M, N, nz = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    off = ctypes.c_long()
    rc = L.ref_mm_read_header(str(path).encode(), ctypes.byref(M), ctypes.byref(N), ctypes.byref(nz),
                              ctypes.byref(off))
    return rc, M.value, N.value, nz.value, off.value


@pytest.mark.parametrize("binary", [False, True])
def test_round_trip_is_exact(tmp_path, binary):
    st, lens, w = _case()
    p = str(tmp_path / ("w.bmtx" if binary else "w.mtx"))
    R.write_weights_file(p, st, w, st_len=lens, binary=binary)
    back = R.read_weights_file(p, st, st_len=lens, binary=binary)
    assert np.array_equal(back, w)


@pytest.mark.parametrize("binary", [False, True])
def test_header_and_entries_as_the_reference_reads_them(tmp_path, binary):
    L = _ref_mmio()
    st, lens, w = _case(N=200, n_pad=9, seed=1)
    p = tmp_path / "w.mtx"
    R.write_weights_file(str(p), st, w, st_len=lens, binary=binary)
    rc, M, N, nz, off = _ref_header(L, p)
    assert rc == 0 and (M, N, nz) == (200, 200, int(lens.sum()))
    raw = p.read_bytes()[off:]
    rows = np.concatenate([np.full(l, i + 1) for i, l in enumerate(lens)])
    cols = np.concatenate([st[i, :l] + 1 for i, l in enumerate(lens)])
    vals = np.concatenate([w[i, :l] for i, l in enumerate(lens)])
    if binary:  # raw int, int, double records (rbffd.cpp:1360-1365)
        rec = np.frombuffer(raw, dtype=np.dtype([("i", "<i4"), ("j", "<i4"), ("v", "<f8")]))
        assert len(rec) == nz
        assert np.array_equal(rec["i"], rows) and np.array_equal(rec["j"], cols) and np.array_equal(rec["v"], vals)
    else:  # "%d %d %24.16le" per entry (rbffd.cpp:1305-1308)
        lines = raw.decode().splitlines()
        assert len(lines) == nz
        expect = ["%d %d %24.16e" % (a, b, c) for a, b, c in zip(rows, cols, vals)]
        assert lines == expect


@pytest.mark.parametrize("binary", [False, True])
def test_reads_a_file_with_the_reference_header(tmp_path, binary):
    """Header written by the reference's mmio, entries in its forms."""
    L = _ref_mmio()
    st, lens, w = _case(N=150, n_pad=10, seed=2)
    p = tmp_path / "ref.mtx"
    nz = int(lens.sum())
    L.ref_mm_write_header(str(p).encode(), 150, 150, nz)
    with open(p, "ab") as f:
        for i in range(150):
            for j in range(lens[i]):
                if binary:
                    f.write(np.array([i + 1, st[i, j] + 1], dtype="<i4").tobytes() + np.float64(w[i, j]).tobytes())
                else:
                    f.write(("%d %d %24.16e\n" % (i + 1, st[i, j] + 1, w[i, j])).encode())
    assert np.array_equal(R.read_weights_file(str(p), st, st_len=lens, binary=binary), w)


def test_refuses_files_for_other_stencils(tmp_path):
    st, lens, w = _case(N=100, n_pad=8, seed=3)
    p = str(tmp_path / "w.mtx")
    R.write_weights_file(p, st, w, st_len=lens, binary=False)
    other = st.copy()
    other[7, 2], other[7, 3] = other[7, 3], other[7, 2]  # same nodes, different order
    with pytest.raises(R.RbffdError):
        R.read_weights_file(p, other, st_len=lens, binary=False)
    with pytest.raises(R.RbffdError):  # different stencil count
        R.read_weights_file(p, st[:99], st_len=lens[:99], binary=False)
    with pytest.raises(R.RbffdError):  # wrong form
        R.read_weights_file(p, st, st_len=lens, binary=True)
    text = open(p).read().splitlines()
    with open(p, "w") as f:  # truncated
        f.write("\n".join(text[:-5]) + "\n")
    with pytest.raises(R.RbffdError):
        R.read_weights_file(p, st, st_len=lens, binary=False)
    with pytest.raises(R.RbffdError):
        R.read_weights_file(str(tmp_path / "missing.mtx"), st, st_len=lens)


@pytest.mark.gpu
def test_rbffd_write_and_load_through_the_grid(ctx, tmp_path):
    """RBFFD.writeToFile / loadFromFile (rbffd.h:400-410): device weights to a
    file and back into a fresh grid, bit for bit, both forms."""
    N, n = 3000, 31
    xyz = R.fibonacci_nodes(N, 9)
    st = R.knn_stencils(xyz, n)
    g = R.Grid(ctx, xyz, st)
    der = R.RBFFD(R.LAMBDA | R.LSFC, g, 2)
    der.setEpsilon(0.25 / np.sqrt(4 * np.pi / N))
    der.setPolynomialDegree(2)
    der.computeAllWeightsForAllStencils()
    g2 = R.Grid(ctx, xyz, st)
    der2 = R.RBFFD(R.LAMBDA | R.LSFC, g2, 2)
    for ascii_form, t in ((1, R.LAMBDA), (0, R.LSFC)):
        der.setAsciiWeights(ascii_form)
        der2.setAsciiWeights(ascii_form)
        p = str(tmp_path / ("w_%d.mtx" % t))
        der.writeToFile(t, p)
        der2.loadFromFile(t, p)
        assert np.array_equal(der2.getWeights(t), der.getWeights(t))
    g.close()
    g2.close()
