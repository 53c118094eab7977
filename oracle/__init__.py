"""ctypes bindings for the oracle -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg (and its ``--impl reference`` arm) may import this package, and only as
the checker or the timed CPU baseline.  The product package never imports it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = {}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)

# DerType bit values (src/rbffd/rbffd.h:43-60)
X, Y, Z, LAPL, R, HV, LAMBDA, THETA = 0x1, 0x2, 0x4, 0x8, 0x10, 0x20, 0x40, 0x80
LSFC, XSFC, YSFC, ZSFC, INTERP = 0x100, 0x200, 0x400, 0x800, 0x8000


def _p(a, t=_dp):
    return None if a is None else a.ctypes.data_as(t)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "_build", "liboracle.so")
        if not os.path.exists(path):
            from . import build as _b
            _b.build_oracle()
        L = ctypes.CDLL(path)
        L.orc_rbf.restype = ctypes.c_double
        L.orc_rbf.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                              ctypes.c_double, ctypes.c_int]
        L.orc_lu_solve.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, _dp]
        L.orc_poly_size.argtypes = [ctypes.c_int]
        L.orc_cart2sph.argtypes = [ctypes.c_double] * 3 + [_dp, _dp]
        L.orc_cart2sph.restype = None
        L.orc_weights.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _ip, _ip, _dp, ctypes.c_uint, ctypes.c_int,
                                  ctypes.c_int, _ip, ctypes.c_int, ctypes.c_double, _dp, ctypes.c_int]
        L.orc_assemble.argtypes = [_dp, _ip, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_uint,
                                   ctypes.c_int, ctypes.c_int, _dp]
        L.orc_apply.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, _dp, ctypes.c_int, _dp, _dp, ctypes.c_int,
                                ctypes.c_int, ctypes.c_int]
        L.orc_apply.restype = None
        L.orc_cosine_bell_coeffs.argtypes = [ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             _dp, _dp]
        L.orc_cosine_bell_coeffs.restype = None
        L.orc_rk4_advect.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, _dp, _dp, _dp, _dp, _dp, ctypes.c_int,
                                     _dp, ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.orc_rk4_heat.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, _dp, ctypes.c_double, ctypes.c_int, _dp,
                                   ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.orc_set_fused.argtypes = [ctypes.c_int]
        L.orc_set_fused.restype = None
        L.orc_nodes_fibonacci.argtypes = [ctypes.c_int, ctypes.c_uint64, _dp]
        L.orc_sph_heat.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double, _dp]
        _LIB = L
    return _LIB


def ref_lib(name):
    """Reference code compiled from its own sources (oracle/_ref), or None if absent."""
    if name not in _REF:
        path = os.path.join(HERE, "_ref", "lib%s.so" % name)
        _REF[name] = ctypes.CDLL(path) if os.path.exists(path) else None
        L = _REF[name]
        if L is not None and name == "ref_rbf":
            L.ref_rbf.restype = ctypes.c_double
            L.ref_rbf.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_int]
            L.ref_cart2sph.argtypes = [ctypes.c_double] * 3 + [_dp] * 3
            L.ref_cart2sph.restype = None
        if L is not None and name == "ref_kdtree":
            L.ref_knn.argtypes = [_dp, ctypes.c_int, ctypes.c_int, _ip, _dp]
        if L is not None and name == "ref_grid":
            L.ref_stencils_hash.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            _dp, ctypes.c_double, _dp, _ip, _ip]
            L.ref_stencils_generate.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, _ip, _ip]
        if L is not None and name == "ref_norms":
            L.ref_sol_norms.argtypes = [_dp, _dp, ctypes.c_int, _dp]
            L.ref_sol_norms.restype = None
        if L is not None and name == "ref_rbffd":
            L.ref_rbffd_create.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_int, ctypes.c_double, ctypes.c_int, _ip,
                                           ctypes.POINTER(ctypes.c_void_p)]
            L.ref_rbffd_destroy.argtypes = [ctypes.c_void_p]
            L.ref_rbffd_destroy.restype = None
            L.ref_rbffd_weights.argtypes = [ctypes.c_void_p, ctypes.c_uint, _dp]
            L.ref_rbffd_system.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
            L.ref_rbffd_apply.argtypes = [ctypes.c_void_p, ctypes.c_uint, _dp, _dp, ctypes.c_int, ctypes.c_int]
            L.ref_rbffd_rk4.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp]
            L.ref_exact_advection.argtypes = [_dp, ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp]
            L.ref_exact_advection.restype = None
        if L is not None and name == "ref_mmio":
            L.ref_mm_write_header.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
            L.ref_mm_read_header.argtypes = [ctypes.c_char_p, _ip, _ip, _ip, ctypes.POINTER(ctypes.c_long)]
    return _REF[name]


class reference_arithmetic:
    """Within this block the oracle's time-stepping arithmetic (SpMV, RK4
    axpys, advection right-hand side) rounds every product and every sum, in
    the reference's source order: the arithmetic of the reference as its own
    build compiles it (x86-64, no FMA).  Outside it, each of those
    multiply-adds is fused: the device kernels' FP64 arithmetic."""

    def __enter__(self):
        lib().orc_set_fused(0)
        return self

    def __exit__(self, *exc):
        lib().orc_set_fused(1)
        return False


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def popcount(v):
    return bin(v & 0xFFFF).count("1")


def types_in_order(der_types):
    return [1 << b for b in range(16) if der_types & (1 << b)]


def weights(xyz, st, st_len, eps, der_types, dim=2, poly_deg=0, hv_k=4, hv_scale=1.0, deg_per_row=None,
            nthreads=0):
    """FP64 weights for every stencil: returns {der_type: array [N, n_pad]}."""
    xyz = _c(xyz, np.float64)
    st = _c(st, np.int32)
    N, n_pad = st.shape
    st_len = None if st_len is None else _c(st_len, np.int32)
    eps = np.full(N, float(eps)) if np.isscalar(eps) else _c(eps, np.float64)
    dpr = None if deg_per_row is None else _c(deg_per_row, np.int32)
    K = popcount(der_types)
    out = np.zeros((K, N, n_pad))
    rc = lib().orc_weights(N, _p(xyz), n_pad, _p(st, _ip), _p(st_len, _ip), _p(eps), der_types, dim, poly_deg,
                           _p(dpr, _ip), hv_k, hv_scale, _p(out), nthreads)
    if rc != 0:
        raise RuntimeError("oracle weight solve hit a zero pivot at row %d" % (-rc - 1))
    return {t: out[k] for k, t in enumerate(types_in_order(der_types))}


def assemble(xyz, stencil, deg, eps, der_types, dim=2, hv_k=4):
    stencil = _c(stencil, np.int32)
    n = len(stencil)
    m = n + lib().orc_poly_size(deg)
    K = popcount(der_types)
    a = np.zeros((m, m + K))
    lib().orc_assemble(_p(_c(xyz, np.float64)), _p(stencil, _ip), n, deg, eps, der_types, dim, hv_k, _p(a))
    return a


def lu_solve(A, B):
    A = _c(A, np.float64)
    B = _c(B, np.float64)
    if B.ndim == 1:
        B = B[:, None]
    m, nrhs = B.shape
    X = np.zeros((m, nrhs))
    info = lib().orc_lu_solve(m, nrhs, _p(A), _p(B), _p(X))
    if info:
        raise np.linalg.LinAlgError("singular at %d" % info)
    return X


def apply(st, st_len, w, u, nthreads=0):
    st = _c(st, np.int32)
    N, n_pad = st.shape
    u = _c(u, np.float64)
    T = 1 if u.ndim == 1 else u.shape[1]
    out = np.zeros_like(u)
    lib().orc_apply(N, n_pad, _p(st, _ip), _p(None if st_len is None else _c(st_len, np.int32), _ip),
                    _p(_c(w, np.float64)), T, _p(u), _p(out), 0, N, nthreads)
    return out


def cosine_bell_coeffs(xyz, a=1.0, alpha=np.pi / 2, u0=None, revolution=1.0):
    xyz = _c(xyz, np.float64)
    N = xyz.shape[0]
    if u0 is None:
        u0 = 2.0 * np.pi * a / revolution
    cu = np.zeros(N)
    cv = np.zeros(N)
    lib().orc_cosine_bell_coeffs(N, _p(xyz), a, alpha, u0, _p(cu), _p(cv))
    return cu, cv


def rk4_advect(st, st_len, w_lambda, w_theta, w_hv, cu, cv, u, dt, nsteps, nthreads=0):
    st = _c(st, np.int32)
    N, n_pad = st.shape
    u = np.array(u, dtype=np.float64, order="C", copy=True)
    T = 1 if u.ndim == 1 else u.shape[1]
    hv = None if w_hv is None else _c(w_hv, np.float64)
    rc = lib().orc_rk4_advect(N, n_pad, _p(st, _ip), _p(None if st_len is None else _c(st_len, np.int32), _ip),
                              _p(_c(w_lambda, np.float64)), _p(_c(w_theta, np.float64)), _p(hv),
                              _p(_c(cu, np.float64)), _p(_c(cv, np.float64)), T, _p(u), dt, nsteps, nthreads)
    if rc:
        raise MemoryError("oracle rk4")
    return u


def rk4_heat(st, st_len, w_lsfc, u, dt, nsteps, kappa=1.0, nthreads=0):
    st = _c(st, np.int32)
    N, n_pad = st.shape
    u = np.array(u, dtype=np.float64, order="C", copy=True)
    T = 1 if u.ndim == 1 else u.shape[1]
    rc = lib().orc_rk4_heat(N, n_pad, _p(st, _ip), _p(None if st_len is None else _c(st_len, np.int32), _ip),
                            _p(_c(w_lsfc, np.float64)), kappa, T, _p(u), dt, nsteps, nthreads)
    if rc:
        raise MemoryError("oracle rk4")
    return u


def ref_knn(xyz, k):
    L = ref_lib("ref_kdtree")
    if L is None:
        return None
    xyz = _c(xyz, np.float64)
    N = xyz.shape[0]
    idx = np.zeros((N, k), dtype=np.int32)
    d = np.zeros((N, k))
    if L.ref_knn(_p(xyz), N, k, _p(idx, _ip), _p(d)) != 0:
        raise RuntimeError("reference kd-tree returned a short list")
    return idx, d


def fibonacci_nodes(N, seed):
    """The benchmark's seeded Fibonacci-sphere nodes (N x 3), restated here so
    the CPU arm builds its grid without the product library."""
    xyz = np.zeros((N, 3))
    if lib().orc_nodes_fibonacci(N, seed, _p(xyz)) != 0:
        raise ValueError("orc_nodes_fibonacci: bad arguments")
    return xyz


def sph_heat(xyz, lmax, coeffs, t, kappa=1.0):
    """sum c_lm exp(-kappa l(l+1) t) Y_lm on the unit sphere (real orthonormal
    harmonics, coefficients ordered l, m = -l..l): the heat workload's initial
    state (t = 0) and exact solution."""
    xyz = _c(xyz, np.float64)
    coeffs = _c(coeffs, np.float64)
    if coeffs.size != (lmax + 1) ** 2:
        raise ValueError("need (lmax+1)^2 coefficients")
    u = np.zeros(xyz.shape[0])
    if lib().orc_sph_heat(xyz.shape[0], _p(xyz), lmax, _p(coeffs), kappa, t, _p(u)) != 0:
        raise ValueError("orc_sph_heat failed")
    return u


def knn_for_baseline(xyz, k):
    """k-nearest stencils for the CPU arm: the reference's own k-d tree
    (external/kdtree/KDTree.h compiled in oracle/_ref) when it was built,
    else scipy's k-d tree (same lists wherever no two distances tie).
    Returns (stencils, source)."""
    r = ref_knn(xyz, k)
    if r is not None:
        return r[0], "reference k-d tree (external/kdtree/KDTree.h)"
    from scipy.spatial import cKDTree
    _, idx = cKDTree(xyz).query(xyz, k)
    return idx.astype(np.int32), "scipy cKDTree"


def cart2sph(x, y, z):
    t, p = ctypes.c_double(), ctypes.c_double()
    lib().orc_cart2sph(x, y, z, ctypes.byref(t), ctypes.byref(p))
    return t.value, p.value


def max_threads():
    return lib().orc_max_threads()


def dense_operator(st, st_len, w, w_hv=None):
    """The dense N x N matrix RBFFD::computeEigenvalues builds
    (src/rbffd/rbffd.cpp:724-764): row i holds stencil i's weights at its
    nodes' columns, plus the hyperviscosity weights when given (rbffd.cpp:737-749).
    The sphere has no boundary nodes, so no identity rows."""
    N, n_pad = st.shape
    A = np.zeros((N, N))
    lens = np.full(N, n_pad) if st_len is None else np.asarray(st_len)
    for i in range(N):
        L = lens[i]
        A[i, st[i, :L]] = w[i, :L] + (w_hv[i, :L] if w_hv is not None else 0.0)
    return A


def eigenvalues(A):
    """Every eigenvalue of a dense real matrix: LAPACK dgeev through numpy, the
    routine Armadillo's eig_gen calls (rbffd.cpp:768)."""
    return np.linalg.eigvals(A)


def eig_classify(re, zero_tol=1e-8):
    """Restatement of the classification loop of RBFFD::computeEigenvalues
    (rbffd.cpp:771-858): all four extremes start at |Re(eig(0))|; real parts
    above zero_tol count as positive, below -zero_tol as negative, the rest as
    zero.  Returns (EigenvalueOutput fields as a dict, max_neg_eig -- the
    reference's return value)."""
    re = [float(x) for x in re]
    e0 = abs(re[0])
    o = dict(max_pos_eig=e0, min_pos_eig=e0, max_neg_eig=e0, min_neg_eig=e0, nb_positive=0, nb_negative=0,
             nb_zero=0)
    for e in re:
        if e > zero_tol:
            o["nb_positive"] += 1
            o["max_pos_eig"] = abs(e) if abs(e) > o["max_pos_eig"] else o["max_pos_eig"]
            o["min_pos_eig"] = abs(e) if abs(e) < o["min_pos_eig"] else o["min_pos_eig"]
        elif e < -zero_tol:
            o["nb_negative"] += 1
            o["max_neg_eig"] = abs(e) if abs(e) > o["max_neg_eig"] else o["max_neg_eig"]
            o["min_neg_eig"] = abs(e) if abs(e) < o["min_neg_eig"] else o["min_neg_eig"]
        else:
            o["nb_zero"] += 1
    return o, o["max_neg_eig"]


def morton_order(xyz):
    """The grids' default node order: a 3-D Morton curve of the coordinates
    scaled to 21-bit integers over the bounding box (bits interleaved x, y, z
    from the top), ties by index."""
    xyz = np.asarray(xyz, dtype=np.float64)
    lo, hi = xyz.min(0), xyz.max(0)
    ext = hi - lo
    f = np.where(ext > 0, (xyz - lo) / np.where(ext > 0, ext, 1.0), 0.0)
    q = np.minimum(2097151.0, np.maximum(0.0, f * 2097151.0)).astype(np.uint64)
    code = np.zeros(len(xyz), dtype=np.uint64)
    for b in range(20, -1, -1):
        for a in range(3):
            code = (code << np.uint64(1)) | ((q[:, a] >> np.uint64(b)) & np.uint64(1))
    return np.lexsort((np.arange(len(xyz)), code)).astype(np.int32)


def rcm_order(st, st_len=None):
    """Reverse Cuthill-McKee on the stencil graph, restating the algorithm of
    the reference's reordering utility (tests/util/cuthill_mckee/reorder.h:50-60,
    Boost's cuthill_mckee_ordering: starting node per component by
    find_starting_node's pseudo-peripheral search, neighbours by increasing
    degree; Boost is not in the reference tree, so ties follow (degree, index)
    and neighbour lists are sorted by index).  Pure Python: small graphs."""
    st = np.asarray(st)
    N, n_pad = st.shape
    lens = [n_pad] * N if st_len is None else [int(x) for x in st_len]
    nb = [set() for _ in range(N)]
    for i in range(N):
        for j in st[i, :lens[i]]:
            j = int(j)
            if j != i:
                nb[i].add(j)
                nb[j].add(i)
    adj = [sorted(s) for s in nb]
    deg = [len(a) for a in adj]
    numbered = [False] * N

    def last_level(r):
        seen = {r}
        level = [r]
        ecc = 0
        while True:
            nxt = []
            for v in level:
                for w in adj[v]:
                    if not numbered[w] and w not in seen:
                        seen.add(w)
                        nxt.append(w)
            if not nxt:
                break
            level = nxt
            ecc += 1
        best = level[0]
        for v in level:
            if deg[v] < deg[best]:
                best = v
        return best, ecc

    cm = []
    for v0 in range(N):
        if numbered[v0]:
            continue
        r = v0
        x, ecc_r = last_level(r)
        y, ecc_x = last_level(x)
        while ecc_x > ecc_r:
            r, ecc_r, x = x, ecc_x, y
            y, ecc_x = last_level(x)
        head = len(cm)
        numbered[x] = True
        cm.append(x)
        while head < len(cm):
            v = cm[head]
            head += 1
            fresh = [w for w in adj[v] if not numbered[w]]
            for w in fresh:
                numbered[w] = True
            cm.extend(sorted(fresh, key=lambda w: (deg[w], w)))
    return np.array(cm[::-1], dtype=np.int32)


def ref_stencils_hash(xyz, n, dims=(10, 10, 10), extents=None, max_radius=1.7976931348623157e308):
    """The reference's own Grid::generateStencilsHash (compiled into
    oracle/_ref/libref_grid.so): (node order, stencils [N][n] in the new
    numbering padded with -1, stencil lengths).  The order is recovered by
    matching the re-sorted coordinates to the input (coordinates are unique)."""
    L = ref_lib("ref_grid")
    if L is None:
        return None
    xyz = _c(xyz, np.float64)
    N = len(xyz)
    xs = np.zeros_like(xyz)
    st = np.zeros((N, n), dtype=np.int32)
    ln = np.zeros(N, dtype=np.int32)
    ext = None if extents is None else _c(extents, np.float64)
    rc = L.ref_stencils_hash(_p(xyz), N, n, dims[0], dims[1], dims[2], _p(ext), max_radius, _p(xs), _p(st, _ip),
                             _p(ln, _ip))
    if rc:
        raise RuntimeError("ref_stencils_hash")
    key = {tuple(p): i for i, p in enumerate(xyz.tolist())}
    order = np.array([key[tuple(p)] for p in xs.tolist()], dtype=np.int32)
    return order, st, ln


def ref_stencils_generate(xyz, n, method, max_radius=1.7976931348623157e308):
    """The reference's own Grid::generateStencilsBruteForce (method 0) or
    generateStencilsKDTree (method 1) with max_st_radius trimming (compiled
    into oracle/_ref/libref_grid.so): (stencils [N][n] padded with -1,
    stencil lengths), in the caller's numbering."""
    L = ref_lib("ref_grid")
    if L is None:
        return None
    xyz = _c(xyz, np.float64)
    N = len(xyz)
    st = np.zeros((N, n), dtype=np.int32)
    ln = np.zeros(N, dtype=np.int32)
    if L.ref_stencils_generate(_p(xyz), N, n, int(method), float(max_radius), _p(st, _ip), _p(ln, _ip)):
        raise RuntimeError("ref_stencils_generate")
    return st, ln


def variable_epsilon(xyz, st, st_len, alpha, eps):
    """RBFFD::setVariableEpsilon, VARIABLE_EPS_TYPE 1 (src/rbffd/rbffd.cpp:1389,
    1411-1416) with Grid::computeStencilRadii's max radius
    (src/grids/grid_interface.cpp:556-557): eps[centre] = 1 / (alpha * |x_last
    - x_centre|), the magnitude summed x, y, z left to right."""
    eps = np.array(eps, dtype=np.float64, copy=True)
    for i in range(st.shape[0]):
        ln = st.shape[1] if st_len is None else int(st_len[i])
        c, last = int(st[i, 0]), int(st[i, ln - 1])
        d = xyz[last] - xyz[c]
        eps[c] = 1.0 / (alpha * np.sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]))
    return eps


def alt_sfc(xyz, wx, wy, wz):
    """ALT_XSFC, ALT_YSFC, ALT_ZSFC from the X, Y, Z weights: the projection
    (I - x x^T) at each stencil centre, left to right without fused
    multiply-adds, as RBFFD::computeAllWeightsForStencil_Direct forms them
    (src/rbffd/rbffd.cpp:337-347).  xyz are the centres, w* [N][n]."""
    x, y, z = (np.asarray(xyz)[:, k:k + 1] for k in range(3))
    ax = (1 - x * x) * wx + (-x * y) * wy + (-x * z) * wz
    ay = (-x * y) * wx + (1 - y * y) * wy + (-y * z) * wz
    az = (-x * z) * wx + (-y * z) * wy + (1 - z * z) * wz
    return ax, ay, az


def ref_sol_norms(sol, exact):
    """The reference's own l1/l2/linf norms and calcSolNorms' relative rule
    (oracle/_ref/libref_norms.so): [l1, l1 rel, l2, l2 rel, linf, linf rel]."""
    L = ref_lib("ref_norms")
    out = np.zeros(6)
    sol, exact = _c(sol, np.float64), _c(exact, np.float64)
    L.ref_sol_norms(_p(sol), _p(exact), len(sol), _p(out))
    return out


def vortex_rollup_w(xyz):
    """Angular velocity of VortexRollup::solve (src/pdes/hyperbolic/vortex_rollup.cpp:34-47):
    theta the cart2sph latitude, rho = 3 cos(theta), Vt = (3 sqrt(3)/2)
    sech(rho)^2 tanh(rho), w = Vt / rho (0 where |rho| < 4 eps), with the
    C library's functions through Python's math module."""
    import math
    out = np.zeros(len(xyz))
    c = 3.0 * math.sqrt(3.0) / 2.0
    for i, (x, y, z) in enumerate(np.asarray(xyz).tolist()):
        th = math.atan2(z, math.sqrt(x * x + y * y))
        rho = 3.0 * math.cos(th)
        s = 1.0 / math.cosh(rho)
        vt = c * (s * s) * math.tanh(rho)
        out[i] = 0.0 if abs(rho) < 4.0 * 2.220446049250313e-16 else vt / rho
    return out


def exact_vortex_rollup(xyz, t):
    """ExactRollup::operator() (tests/experiments/vortex_rollup_on_sphere/exact_rollup.h:25-35),
    gamma = 5: h = 1 - tanh((rho / gamma) sin(lambda - w t))."""
    import math
    w = vortex_rollup_w(xyz)
    out = np.zeros(len(xyz))
    for i, (x, y, z) in enumerate(np.asarray(xyz).tolist()):
        rho = 3.0 * math.cos(math.atan2(z, math.sqrt(x * x + y * y)))
        out[i] = 1.0 - math.tanh((rho / 5.0) * math.sin(math.atan2(y, x) - w[i] * t))
    return out


class RefRBFFD:
    """The reference's own RBFFD / TimeDependentPDE / CosineBell / VortexRollup,
    compiled from its sources into oracle/_ref/libref_rbffd.so (see
    oracle/ref_rbffd.cpp): a problem built as the cosine-bell experiment
    builds it on one rank (k-d tree stencils, one subdomain, RBFFD with
    ONE_MONOMIAL: the constant is the only polynomial term)."""

    KIND_COSINE_BELL, KIND_HEAT, KIND_VORTEX = 0, 1, 2

    @staticmethod
    def available():
        return ref_lib("ref_rbffd") is not None

    def __init__(self, xyz, n, der_types, eps, dim=2, hv_k=4, hv_gamma=8e-4, use_hv=False):
        self.L = ref_lib("ref_rbffd")
        if self.L is None:
            raise RuntimeError("oracle/_ref/libref_rbffd.so is not built (needs the reference tree)")
        self.xyz = _c(xyz, np.float64)
        self.N, self.n = self.xyz.shape[0], n
        self.stencils = np.zeros((self.N, n), dtype=np.int32)
        h = ctypes.c_void_p()
        rc = self.L.ref_rbffd_create(_p(self.xyz), self.N, n, der_types, dim, eps, hv_k, hv_gamma,
                                     1 if use_hv else 0, _p(self.stencils, _ip), ctypes.byref(h))
        if rc != 0:
            raise RuntimeError("the reference's RBFFD set-up failed")
        self.h = h

    def weights(self, der_type):
        """Stored weights: N x (n + 1), the stencil weights then the constant's."""
        w = np.zeros((self.N, self.n + 1))
        if self.L.ref_rbffd_weights(self.h, der_type, _p(w)) != 0:
            raise RuntimeError("no weights of type 0x%x" % der_type)
        return w

    def system(self, st_index, n_types):
        """(LHS, RHS) of one stencil from getStencilLHS / getStencilMultiRHS."""
        m = self.n + 1
        A = np.zeros(m * m)
        B = np.zeros(m * n_types)
        self.L.ref_rbffd_system(self.h, st_index, _p(A), _p(B))
        return A.reshape(m, m).T.copy(), B.reshape(n_types, m).T.copy()

    def apply(self, der_type, u, start=0, count=0):
        u = _c(u, np.float64)
        d = np.zeros(self.N)
        self.L.ref_rbffd_apply(self.h, der_type, _p(u), _p(d), start, count)
        return d

    def rk4(self, kind, u, dt, nsteps, a=1.0, alpha=np.pi / 2, revolution=1036800.0, use_hv=True):
        u = np.array(u, dtype=np.float64)
        if self.L.ref_rbffd_rk4(self.h, kind, a, alpha, revolution, 1 if use_hv else 0, dt, nsteps, _p(u)) != 0:
            raise RuntimeError("ref_rbffd_rk4")
        return u

    def close(self):
        if self.h:
            self.L.ref_rbffd_destroy(self.h)
            self.h = None


def ref_exact_advection(xyz, a=1.0, t=0.0):
    """ExactAdvection (tests/experiments/cosine_bell_on_sphere/exact_advection.h)
    compiled from the reference, at the nodes; None without the library."""
    L = ref_lib("ref_rbffd")
    if L is None:
        return None
    xyz = _c(xyz, np.float64)
    out = np.zeros(xyz.shape[0])
    L.ref_exact_advection(_p(xyz), xyz.shape[0], a, t, _p(out))
    return out
