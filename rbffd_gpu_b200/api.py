"""Python view of the C ABI, shaped like the reference classes it replaces.

``RBFFD`` mirrors src/rbffd/rbffd.h (DerType flags, setters,
computeAllWeightsForAllStencils, applyWeightsForDeriv, getStencilWeights);
``TimeDependentPDE`` / ``CosineBell`` mirror src/pdes/time_dependent_pde.h and
src/pdes/hyperbolic/cosine_bell.h (advance(RK4, dt), fillInitialConditions,
getTime).  Every method calls librbffd_sm100.so; errors raise RbffdError with
the library's message.
"""
import ctypes

import numpy as np

from . import _lib

F32, F64 = 0, 1
# FP64 arithmetic of the apply and time-stepping kernels (rbffd_ctx_set_arithmetic):
# fused multiply-adds (default), or rounded products then sums, the reference build's arithmetic
ARITH_FUSED, ARITH_UNFUSED = 0, 1
ELIM_AUTO, ELIM_UNBLOCKED, ELIM_BLOCKED, ELIM_ROW_MAP, ELIM_REGISTERS = 0, 1, 2, 3, 4
X, Y, Z, LAPL, R, HV, LAMBDA, THETA = 0x1, 0x2, 0x4, 0x8, 0x10, 0x20, 0x40, 0x80
LSFC, XSFC, YSFC, ZSFC, INTERP = 0x100, 0x200, 0x400, 0x800, 0x8000
ALT_XSFC, ALT_YSFC, ALT_ZSFC = 0x1000, 0x2000, 0x4000
EULER, MIDPOINT, RK4 = 0, 1, 2  # TimeDependentPDE::TimeScheme (time_dependent_pde.h:20)

ADVANCE_GRAPH, ADVANCE_UNFUSED, ADVANCE_ASYNC, ADVANCE_RESIDENT = 0x1, 0x2, 0x4, 0x8
RHS_COSINE_BELL, RHS_HEAT, RHS_ADVECTION = 1, 2, 3


class RbffdError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s (%d): %s" % (_lib.load().rbffd_status_string(status).decode(), status, message))
        self.status = status


def _dp(a):
    return None if a is None else a.ctypes.data_as(_lib.dp)


def _ip(a):
    return a.ctypes.data_as(_lib.ip)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def version():
    return _lib.load().rbffd_version().decode()


def device_count():
    n = ctypes.c_int(0)
    rc = _lib.load().rbffd_device_count(ctypes.byref(n))
    return n.value if rc == 0 else 0


# ---------------------------------------------------------------------------
# host-side inputs

def fibonacci_nodes(N, seed):
    xyz = np.zeros((N, 3))
    rc = _lib.load().rbffd_nodes_fibonacci(N, seed, _dp(xyz))
    if rc:
        raise RbffdError(rc, "rbffd_nodes_fibonacci")
    return xyz


def knn_stencils(xyz, n, nthreads=0, return_ties=False):
    xyz = _f64(xyz)
    N = xyz.shape[0]
    st = np.zeros((N, n), dtype=np.int32)
    ties = ctypes.c_int(0)
    rc = _lib.load().rbffd_stencils_knn(_dp(xyz), N, n, _ip(st), ctypes.byref(ties), nthreads)
    if rc:
        raise RbffdError(rc, "rbffd_stencils_knn")
    return (st, ties.value) if return_ties else st


ST_BRUTE_FORCE, ST_KDTREE, ST_HASH = 0, 1, 2  # Grid::st_generator_t (grid_interface.h:37)


def generate_stencils(xyz, n, method=ST_BRUTE_FORCE, max_radius=1.7976931348623157e308, nthreads=0):
    """Grid::generateStencils with the reference's default brute-force
    generator or its k-d tree, and max_st_radius trimming: (stencils [N][n],
    lengths [N]), padding the centre.  Host only; ST_HASH is stencils_hash."""
    xyz = _f64(xyz)
    N = xyz.shape[0]
    st = np.zeros((N, n), dtype=np.int32)
    ln = np.zeros(N, dtype=np.int32)
    rc = _lib.load().rbffd_stencils_generate(_dp(xyz), N, n, int(method), float(max_radius), _ip(st), _ip(ln), None,
                                             nthreads)
    if rc:
        raise RbffdError(rc, "rbffd_stencils_generate")
    return st, ln


def generate_stencils_gpu(ctx, xyz, n, method=ST_BRUTE_FORCE, max_radius=1.7976931348623157e308):
    """generate_stencils on ctx's device (identical lists and lengths)."""
    xyz = _f64(xyz)
    N = xyz.shape[0]
    st = np.zeros((N, n), dtype=np.int32)
    ln = np.zeros(N, dtype=np.int32)
    ctx.check(ctx.L.rbffd_stencils_generate_gpu(ctx.h, _dp(xyz), N, n, int(method), float(max_radius), _ip(st), _ip(ln),
                                                None), "rbffd_stencils_generate_gpu")
    return st, ln


def variable_epsilon(xyz, stencils, st_len, alpha, eps=None):
    """RBFFD::setVariableEpsilon's per-stencil eps (rbffd.cpp:1378-1420):
    eps[centre] = 1 / (alpha * distance to the stencil's last node); entries
    of eps (default ones) at nodes that centre no stencil are kept.  Host only."""
    xyz, st = _f64(xyz), _i32(stencils)
    N, n_pad = st.shape
    out = np.ones(len(xyz)) if eps is None else np.array(eps, dtype=np.float64, copy=True)
    rc = _lib.load().rbffd_variable_epsilon(N, _dp(xyz), n_pad, _ip(st), None if st_len is None else _ip(_i32(st_len)),
                                            float(alpha), _dp(out))
    if rc:
        raise RbffdError(rc, "rbffd_variable_epsilon")
    return out


def write_weights_file(filename, stencils, w, st_len=None, binary=True):
    """The reference's weight file (Matrix Market, text or binary form) for
    weights w [N][n_pad] of stencils [N][n_pad]; host only."""
    st = _i32(stencils)
    w = _f64(w)
    N, n_pad = st.shape
    sl = None if st_len is None else _i32(st_len)
    rc = _lib.load().rbffd_weights_file_write(filename.encode(), int(binary), N, n_pad, _ip(st),
                                              None if sl is None else _ip(sl), _dp(w))
    if rc:
        raise RbffdError(rc, "rbffd_weights_file_write(%s)" % filename)


def read_weights_file(filename, stencils, st_len=None, binary=True):
    """Weights [N][n_pad] from the reference's weight file for these stencils; host only."""
    st = _i32(stencils)
    N, n_pad = st.shape
    sl = None if st_len is None else _i32(st_len)
    w = np.zeros((N, n_pad))
    rc = _lib.load().rbffd_weights_file_read(filename.encode(), int(binary), N, n_pad, _ip(st),
                                             None if sl is None else _ip(sl), _dp(w))
    if rc:
        raise RbffdError(rc, "rbffd_weights_file_read(%s)" % filename)
    return w


def vortex_rollup_coefficients(xyz):
    """w(theta) of VortexRollup::solve per node (vortex_rollup.cpp:34-47)."""
    xyz = _f64(xyz)
    w = np.zeros(len(xyz))
    rc = _lib.load().rbffd_vortex_rollup_coefficients(len(xyz), _dp(xyz), _dp(w))
    if rc:
        raise RbffdError(rc, "rbffd_vortex_rollup_coefficients")
    return w


def exact_vortex_rollup(xyz, t):
    """ExactRollup (exact_rollup.h:25-35)."""
    xyz = _f64(xyz)
    h = np.zeros(len(xyz))
    rc = _lib.load().rbffd_exact_vortex_rollup(len(xyz), _dp(xyz), float(t), _dp(h))
    if rc:
        raise RbffdError(rc, "rbffd_exact_vortex_rollup")
    return h


NORM_NAMES = ("l1", "l1_rel", "l2", "l2_rel", "linf", "linf_rel")


def sol_norms(sol, exact):
    """PDE::calcSolNorms (pde.cpp:467-510): absolute and relative l1, l2, linf errors."""
    sol, exact = _f64(sol).ravel(), _f64(exact).ravel()
    out = np.zeros(6)
    rc = _lib.load().rbffd_sol_norms(_dp(sol), _dp(exact), len(sol), _dp(out))
    if rc:
        raise RbffdError(rc, "rbffd_sol_norms")
    return dict(zip(NORM_NAMES, out.tolist()))


def stencils_hash(xyz, n, dims=(10, 10, 10), extents=None, max_radius=1.7976931348623157e308):
    """Grid::generateStencilsHash (the cosine-bell experiment's generator):
    (order, stencils, lengths), the stencils in the new numbering where node
    order[k] is placed at k.  Host only."""
    xyz = _f64(xyz)
    N = len(xyz)
    order = np.zeros(N, dtype=np.int32)
    st = np.zeros((N, n), dtype=np.int32)
    ln = np.zeros(N, dtype=np.int32)
    ext = None if extents is None else _f64(extents)
    rc = _lib.load().rbffd_stencils_hash(_dp(xyz), N, n, int(dims[0]), int(dims[1]), int(dims[2]),
                                         None if ext is None else _dp(ext), float(max_radius), _ip(order), _ip(st),
                                         _ip(ln))
    if rc:
        raise RbffdError(rc, "rbffd_stencils_hash")
    return order, st, ln


ORDER_MORTON, ORDER_RCM, ORDER_GIVEN = 0, 1, 2


def node_order(method, xyz=None, stencils=None, st_len=None):
    """The node order a grid can use (reorder.h's `order`: order[k] is the
    node placed at position k): ORDER_MORTON (needs xyz), ORDER_RCM (reverse
    Cuthill-McKee on the stencil graph; needs stencils) or ORDER_GIVEN.  Host only."""
    st = None if stencils is None else _i32(stencils)
    N = len(xyz) if xyz is not None else st.shape[0]
    n_pad = 0 if st is None else st.shape[1]
    order = np.zeros(N, dtype=np.int32)
    rc = _lib.load().rbffd_node_order(N, None if xyz is None else _dp(_f64(xyz)), n_pad,
                                      None if st is None else _ip(st), None if st_len is None else _ip(_i32(st_len)),
                                      int(method), _ip(order))
    if rc:
        raise RbffdError(rc, "rbffd_node_order")
    return order


def hessenberg_eigenvalues(H):
    """Eigenvalues of a real upper Hessenberg matrix (the Arnoldi check's
    projected problem; shifted QR in complex arithmetic, host only)."""
    H = _f64(H)
    n = H.shape[0]
    re, im = np.zeros(n), np.zeros(n)
    rc = _lib.load().rbffd_hessenberg_eigenvalues(n, _dp(H), _dp(re), _dp(im))
    if rc:
        raise RbffdError(rc, "rbffd_hessenberg_eigenvalues")
    return re + 1j * im


def eig_output_dict(o):
    return {k: getattr(o, k) for k, _ in _lib.EigOutput._fields_}


def eig_classify(re, zero_tol=1e-8):
    """The reference's classification of eigenvalue real parts
    (rbffd.cpp:781-858): (EigenvalueOutput as a dict, max |Re| of the negative
    ones).  Host only."""
    re = _f64(re)
    o = _lib.EigOutput()
    ret = ctypes.c_double()
    rc = _lib.load().rbffd_eig_classify(_dp(re), re.size, float(zero_tol), ctypes.byref(o), ctypes.byref(ret))
    if rc:
        raise RbffdError(rc, "rbffd_eig_classify")
    return eig_output_dict(o), ret.value


def knn_stencils_gpu(ctx, xyz, n, return_ties=False):
    """The stencils of knn_stencils (identical lists), searched on ctx's device."""
    xyz = _f64(xyz)
    N = xyz.shape[0]
    st = np.zeros((N, n), dtype=np.int32)
    ties = ctypes.c_int(0)
    ctx.check(ctx.L.rbffd_stencils_knn_gpu(ctx.h, _dp(xyz), N, n, _ip(st), ctypes.byref(ties)), "rbffd_stencils_knn_gpu")
    return (st, ties.value) if return_ties else st


def exact_cosine_bell(xyz, a=1.0):
    xyz = _f64(xyz)
    h = np.zeros(xyz.shape[0])
    rc = _lib.load().rbffd_exact_cosine_bell(xyz.shape[0], _dp(xyz), a, _dp(h))
    if rc:
        raise RbffdError(rc, "rbffd_exact_cosine_bell")
    return h


def exact_sph_heat(xyz, lmax, coeffs, t, kappa=1.0):
    xyz = _f64(xyz)
    coeffs = _f64(coeffs)
    if coeffs.size != (lmax + 1) ** 2:
        raise ValueError("need (lmax+1)^2 coefficients")
    u = np.zeros(xyz.shape[0])
    rc = _lib.load().rbffd_exact_sph_heat(xyz.shape[0], _dp(xyz), lmax, _dp(coeffs), kappa, t, _dp(u))
    if rc:
        raise RbffdError(rc, "rbffd_exact_sph_heat")
    return u


# ---------------------------------------------------------------------------

class Context:
    """One CUDA device, one stream; owns every device buffer made from it."""

    def __init__(self, device=0):
        self.L = _lib.load()
        h = ctypes.c_void_p()
        rc = self.L.rbffd_ctx_create(device, ctypes.byref(h))
        if rc:
            raise RbffdError(rc, "rbffd_ctx_create(device=%d)" % device)
        self.h = h
        self.device = device

    def check(self, rc, what=""):
        if rc:
            raise RbffdError(rc, "%s: %s" % (what, self.L.rbffd_ctx_last_error(self.h).decode()))

    def synchronize(self):
        self.check(self.L.rbffd_ctx_synchronize(self.h), "synchronize")

    def mem_info(self):
        held, free, total = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t()
        self.check(self.L.rbffd_ctx_mem_info(self.h, ctypes.byref(held), ctypes.byref(free), ctypes.byref(total)))
        return held.value, free.value, total.value

    def setArithmetic(self, arith):
        """FP64 arithmetic of rbffd_apply* calls and of FP64 one-tracer PDEs
        created afterwards: ARITH_FUSED, or ARITH_UNFUSED (the reference's own
        build: a rounded product, then a rounded sum)."""
        self.check(self.L.rbffd_ctx_set_arithmetic(self.h, arith), "set_arithmetic")

    def getArithmetic(self):
        a = ctypes.c_int()
        self.check(self.L.rbffd_ctx_get_arithmetic(self.h, ctypes.byref(a)))
        return a.value

    def setWeightsElimination(self, method):
        """Elimination of the batched weight solves on this context: ELIM_AUTO
        (autotuned per system size), ELIM_UNBLOCKED, ELIM_BLOCKED, ELIM_ROW_MAP
        or ELIM_REGISTERS; every method gives the same weights bit for bit."""
        self.check(self.L.rbffd_weights_set_elimination(self.h, method), "set_elimination")

    def getWeightsElimination(self):
        a = ctypes.c_int()
        self.check(self.L.rbffd_weights_get_elimination(self.h, ctypes.byref(a)))
        return a.value

    def stream(self):
        s = ctypes.c_void_p()
        self.check(self.L.rbffd_ctx_stream(self.h, ctypes.byref(s)))
        return s.value

    def close(self):
        if getattr(self, "h", None):
            self.L.rbffd_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Grid:
    """Nodes and stencils (the reference Grid: getNodeList, getStencils, getMaxStencilSize)."""

    def __init__(self, ctx, nodes, stencils, st_len=None, global_nodes=None, order=None):
        """order: the internal node order (ORDER_MORTON by default, ORDER_RCM or ORDER_GIVEN)."""
        self.ctx = ctx
        self.nodes = _f64(nodes)
        self.stencils = _i32(stencils)
        self.N, self.n_pad = self.stencils.shape
        self.st_len = None if st_len is None else _i32(st_len)
        self.global_nodes = global_nodes or self.N
        h = ctypes.c_void_p()
        ctx.check(ctx.L.rbffd_grid_create_ordered(ctx.h, self.N, _dp(self.nodes), self.n_pad, _ip(self.stencils),
                                                  None if self.st_len is None else _ip(self.st_len),
                                                  ORDER_MORTON if order is None else int(order), ctypes.byref(h)),
                  "rbffd_grid_create")
        self.h = h

    def getNodeList(self):
        return self.nodes

    def getStencils(self):
        return self.stencils

    def getStencilsSize(self):
        return self.N

    def getNodeListSize(self):
        return self.N

    def getGlobalNodeListSize(self):
        return self.global_nodes

    def getMaxStencilSize(self):
        return self.n_pad

    def nbytes(self):
        b = ctypes.c_size_t()
        self.ctx.check(self.ctx.L.rbffd_grid_nbytes(self.h, ctypes.byref(b)))
        return b.value

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.rbffd_grid_destroy(self.h)
            self.h = None


class RBFFD:
    """Mirror of class RBFFD (src/rbffd/rbffd.h:29-547) on the device."""
    X, Y, Z, LAPL, R, HV, LAMBDA, THETA = X, Y, Z, LAPL, R, HV, LAMBDA, THETA
    LSFC, XSFC, YSFC, ZSFC, INTERP = LSFC, XSFC, YSFC, ZSFC, INTERP
    ALT_XSFC, ALT_YSFC, ALT_ZSFC = ALT_XSFC, ALT_YSFC, ALT_ZSFC

    def __init__(self, typesToCompute, grid, dim_num, rank=0):
        self.computedTypes = typesToCompute
        self.grid = grid
        self.dim_num = dim_num
        self.rank = rank
        self.hv_k, self.hv_gamma = 2, 8e-4  # ctor defaults (rbffd.cpp:26)
        self.useHyperviscosity = 0
        self.var_epsilon = np.ones(grid.N)
        self.poly_deg = 0  # ONE_MONOMIAL (rbffd.cpp:1)
        self.asciiWeights = 0  # binary weight files unless setAsciiWeights(1)
        self.deg_per_row = None

    # -- parameters (rbffd.h:213-381) --
    def setUseHyperviscosity(self, tf):
        self.useHyperviscosity = int(tf)
        self.computedTypes = (self.computedTypes | HV) if tf else (self.computedTypes & ~HV)

    def appendDerTypes(self, t):
        self.computedTypes |= t

    def setHVScalars(self, k, gamma_c):
        self.hv_k, self.hv_gamma = int(k), float(gamma_c)
        return self.hv_gamma

    def getHVScalar(self):
        return -self.hv_gamma * float(self.grid.getGlobalNodeListSize()) ** (-self.hv_k)

    def setEpsilon(self, eps):
        if np.isscalar(eps):
            self.var_epsilon[:] = float(eps)
        else:
            eps = _f64(eps)
            if eps.shape != self.var_epsilon.shape:
                raise ValueError("length of support params list does not match")
            self.var_epsilon = eps.copy()

    def setEpsilonByParameters(self, c1, c2):
        self.setEpsilon(c1 * np.sqrt(self.grid.getGlobalNodeListSize()) - c2)

    def setVariableEpsilon(self, alpha=1.0, beta=1.0):
        """rbffd.cpp:1378-1420 (Sarler 2006): eps at each centre =
        1 / (alpha * distance to the stencil's last node); beta is unused
        there, as in the reference."""
        g = self.grid
        self.var_epsilon = variable_epsilon(g.nodes, g.stencils, g.st_len, alpha, self.var_epsilon)

    def setPolynomialDegree(self, deg, deg_per_row=None):
        """Beyond the reference (which fixes np = 1): -1 none, 0 constant, 1..4."""
        self.poly_deg = int(deg)
        self.deg_per_row = None if deg_per_row is None else _i32(deg_per_row)

    # -- weights --
    def adjustForSFCTypes(self):
        """rbffd.h:507-522: any ALT_*SFC type brings X, Y, Z and all three ALT types."""
        if self.computedTypes & (ALT_XSFC | ALT_YSFC | ALT_ZSFC):
            self.computedTypes |= X | Y | Z | ALT_XSFC | ALT_YSFC | ALT_ZSFC
            return True
        return False

    def computeAllWeightsForAllStencils(self):
        self.adjustForSFCTypes()
        ctx = self.grid.ctx
        p = _lib.WeightParams(self.computedTypes, self.dim_num, self.poly_deg, self.hv_k, self.hv_gamma,
                              float(self.grid.getGlobalNodeListSize()))
        ctx.check(ctx.L.rbffd_weights_compute(self.grid.h, ctypes.byref(p), _dp(self.var_epsilon), 0.0,
                                              None if self.deg_per_row is None else _ip(self.deg_per_row)),
                  "rbffd_weights_compute")

    def setWeights(self, which, w):
        w = _f64(w)
        ctx = self.grid.ctx
        ctx.check(ctx.L.rbffd_weights_set(self.grid.h, which, _dp(w)), "rbffd_weights_set")

    def getWeights(self, which):
        w = np.zeros((self.grid.N, self.grid.n_pad))
        ctx = self.grid.ctx
        ctx.check(ctx.L.rbffd_weights_get(self.grid.h, which, _dp(w)), "rbffd_weights_get")
        return w

    # -- weight files (rbffd.h:400-410; rbffd.cpp:973-1375) --
    def setAsciiWeights(self, binary_or_ascii):
        """1: text Matrix Market files; 0: the binary form (the reference's default)."""
        self.asciiWeights = int(binary_or_ascii)

    def writeToFile(self, which, filename):
        g = self.grid
        w = self.getWeights(which)
        rc = g.ctx.L.rbffd_weights_file_write(filename.encode(), 0 if self.asciiWeights else 1,
                                              g.N, g.n_pad, _ip(g.stencils),
                                              None if g.st_len is None else _ip(g.st_len), _dp(w))
        if rc:
            raise RbffdError(rc, "writeToFile(%s)" % filename)

    def loadFromFile(self, which, filename):
        g = self.grid
        w = np.zeros((g.N, g.n_pad))
        rc = g.ctx.L.rbffd_weights_file_read(filename.encode(), 0 if self.asciiWeights else 1,
                                             g.N, g.n_pad, _ip(g.stencils),
                                             None if g.st_len is None else _ip(g.st_len), _dp(w))
        if rc:
            raise RbffdError(rc, "loadFromFile(%s)" % filename)
        self.setWeights(which, w)

    def getStencilWeights(self, which, st_indx):
        return self.getWeights(which)[st_indx]

    # -- eigenvalue stability check (rbffd.h:281,412-417; rbffd.cpp:703-873) --
    def computeEigenvalues(self, which, exit_on_fail=False, output=None, return_eigenvalues=False):
        """Every eigenvalue of the dense operator `which` (+ HV when
        hyperviscosity is on), classified as the reference does; returns the
        reference's value, max |Re| among the negative eigenvalues (and the
        complex eigenvalues when asked).  `output`, if a dict, receives the
        EigenvalueOutput fields.  Where the reference exits (both signs
        present, or more than one eigenvalue within 1e-8 of zero) this raises
        RbffdError when exit_on_fail."""
        g = self.grid
        re, im = np.zeros(g.N), np.zeros(g.N)
        o = _lib.EigOutput()
        ret = ctypes.c_double()
        g.ctx.check(g.ctx.L.rbffd_eigenvalues(g.h, which, int(bool(self.useHyperviscosity)), _dp(re), _dp(im),
                                              ctypes.byref(o), ctypes.byref(ret)), "rbffd_eigenvalues")
        res = eig_output_dict(o)
        self.cachedEigenvalues = res
        if output is not None:
            output.update(res)
        if exit_on_fail and ((res["nb_negative"] > 0 and res["nb_positive"] > 0) or res["nb_zero"] > 1):
            raise RbffdError(-1, "computeEigenvalues: eigenvalues of both signs or more than one zero: %r" % res)
        return (ret.value, re + 1j * im) if return_eigenvalues else ret.value

    def computeRightmostEigenvalues(self, which, nev=6, ncv=40, tol=1e-8, max_restarts=3000, seed=1):
        """The nev rightmost eigenvalues of `which` (+ HV when hyperviscosity
        is on) by implicitly restarted Arnoldi on the device's sparse operator
        (rbffd_eigen_rightmost): the stability verdict of computeEigenvalues
        for grids too large for the dense check.  Returns a dict with the
        eigenvalues (complex, rightmost first), their residual estimates, how
        many converged, restarts and operator applications."""
        g = self.grid
        re, im, rs = np.zeros(nev), np.zeros(nev), np.zeros(nev)
        nconv, restarts, mv = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        g.ctx.check(g.ctx.L.rbffd_eigen_rightmost(g.h, which, int(bool(self.useHyperviscosity)), nev, ncv, tol,
                                                  max_restarts, seed, _dp(re), _dp(im), _dp(rs), ctypes.byref(nconv),
                                                  ctypes.byref(restarts), ctypes.byref(mv)), "rbffd_eigen_rightmost")
        return {"eigenvalues": re + 1j * im, "residual_estimates": rs, "nconv": nconv.value,
                "restarts": restarts.value, "matvecs": mv.value}

    def getEigenvalues(self):
        if getattr(self, "cachedEigenvalues", None) is None:
            self.computeEigenvalues(LAPL, False)
        return self.cachedEigenvalues

    # -- apply (rbffd.h:257-274) --
    def applyWeightsForDeriv(self, which, u, deriv=None, isChangedU=True, start_indx=0, nb_stencils=None, dtype=F64):
        u = _f64(u)
        N = self.grid.N
        if nb_stencils is None:
            nb_stencils = N - start_indx
        if deriv is None:
            deriv = np.zeros(N)
        ctx = self.grid.ctx
        ctx.check(ctx.L.rbffd_apply(self.grid.h, which, dtype, start_indx, nb_stencils, _dp(u), _dp(deriv)),
                  "rbffd_apply")
        return deriv

    def applyWeightsForDerivDev(self, which, u_ptr, out_ptr, dtype=F64, ntracers=1):
        ctx = self.grid.ctx
        ctx.check(ctx.L.rbffd_apply_dev(self.grid.h, which, dtype, ntracers, u_ptr, out_ptr), "rbffd_apply_dev")


class TimeDependentPDE:
    """Device-resident TimeDependentPDE (src/pdes/time_dependent_pde.h:9-126)."""

    def __init__(self, grid, der, params):
        self.grid, self.der, self.ctx = grid, der, grid.ctx
        self.T = params.ntracers
        self.dtype = params.dtype
        h = ctypes.c_void_p()
        self.ctx.check(self.ctx.L.rbffd_pde_create(grid.h, ctypes.byref(params), ctypes.byref(h)), "rbffd_pde_create")
        self.h = h

    def fillInitialConditions(self, values):
        u = _f64(values).reshape(self.grid.N, self.T) if self.T > 1 else _f64(values)
        self.ctx.check(self.ctx.L.rbffd_pde_set_state(self.h, _dp(np.ascontiguousarray(u))), "set_state")

    def getLocalSolution(self, indx=None):
        """The solution (pde.h:161); one node's value with indx."""
        u = np.zeros((self.grid.N, self.T)) if self.T > 1 else np.zeros(self.grid.N)
        self.ctx.check(self.ctx.L.rbffd_pde_get_state(self.h, _dp(u)), "get_state")
        return u if indx is None else u[indx]

    def syncCPUtoGPU(self):
        """PDE::syncCPUtoGPU (pde.h:166): the device holds the state and every
        read copies it, so there is nothing to synchronise."""

    def setStartEndTime(self, start, end):
        """TimeDependentPDE::setStartEndTime (time_dependent_pde.h:52-56)."""
        self.start_time, self.end_time = float(start), float(end)
        self.setTime(start)

    def checkGlobalError(self, exact, global_grid=None, rel_err_max=-1.0, ignore_sol_error=True):
        """PDE::checkGlobalError (pde.h:130-147): on one rank, checkLocalError."""
        return self.checkLocalError(exact, rel_err_max)

    def advance(self, which=RK4, delta_t=1.0, nsteps=1, graph=False, unfused=False, asynchronous=False,
                resident=False):
        """nsteps RK4 steps (rbffd_pde_advance); resident: all steps in one
        launch of a thread-block cluster holding the operator and state in its
        shared memory (one tracer, small grids)."""
        flags = (ADVANCE_GRAPH if graph else 0) | (ADVANCE_UNFUSED if unfused else 0) | (
            ADVANCE_ASYNC if asynchronous else 0) | (ADVANCE_RESIDENT if resident else 0)
        self.ctx.check(self.ctx.L.rbffd_pde_advance(self.h, which, delta_t, nsteps, flags), "rbffd_pde_advance")

    def checkLocalError(self, exact, rel_err_max=-1.0):
        """PDE::checkLocalError / checkError (pde.h:120-127, pde.cpp:385-465):
        the error norms of the solution against the exact values, printed per
        node group as the reference prints them (the sphere has no boundary
        nodes: the boundary group is empty, the other three are the whole
        grid); returns the whole grid's norms.  Like checkLocalError, a high
        error is reported, never fatal."""
        u = self.getLocalSolution()
        full = sol_norms(u, exact)
        empty = sol_norms(np.zeros(0), np.zeros(0))
        for label, nrm, cnt in (("Boundary", empty, 0), ("Interior Stencils w/o Boundary", full, u.size),
                                ("All Interior", full, u.size), ("Interior & Boundary", full, u.size)):
            for p in ("l1", "l2", "linf"):
                print("%s %s error (%d nodes):   Absolute = %le,    Relative = %le " % (
                    label, p, cnt, nrm[p], nrm[p + "_rel"]))
        if rel_err_max > 0 and full["l2_rel"] > rel_err_max:
            print("[PDE] Error! l2 relative error (=%f%%) is too high to continue. We require %f%% or less." % (
                100.0 * full["l2_rel"], 100.0 * rel_err_max))
        return full

    def setTime(self, t):
        self.ctx.check(self.ctx.L.rbffd_pde_set_time(self.h, t))

    def getTime(self):
        t = ctypes.c_double()
        self.ctx.check(self.ctx.L.rbffd_pde_get_time(self.h, ctypes.byref(t)))
        return t.value

    def setShape(self, lanes_per_row=0, block_threads=0):
        self.ctx.check(self.ctx.L.rbffd_pde_set_shape(self.h, lanes_per_row, block_threads), "set_shape")

    def setArithmetic(self, arith):
        """ARITH_UNFUSED (FP64, one tracer): the reference build's arithmetic,
        one lane per stencil row; ARITH_FUSED: fused multiply-adds, autotuned shape."""
        self.ctx.check(self.ctx.L.rbffd_pde_set_arithmetic(self.h, arith), "set_arithmetic")

    def getArithmetic(self):
        a = ctypes.c_int()
        self.ctx.check(self.ctx.L.rbffd_pde_get_arithmetic(self.h, ctypes.byref(a)))
        return a.value

    def getShape(self):
        """(lanes per row, threads per block, rows per tiled block or 0)."""
        a, b, r = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self.ctx.check(self.ctx.L.rbffd_pde_get_shape(self.h, ctypes.byref(a), ctypes.byref(b)))
        self.ctx.check(self.ctx.L.rbffd_pde_get_tiling(self.h, ctypes.byref(r)))
        return a.value, b.value, r.value

    def setFusedOperator(self, on=True):
        """Advection: one fused operator -(cu Wl + cv Wt) + Whv per stage (formed
        in FP64, rounded to the PDE's dtype; not in the unfused arithmetic)."""
        self.ctx.check(self.ctx.L.rbffd_pde_set_fused_operator(self.h, int(bool(on))), "set_fused_operator")

    def setCompensatedState(self, on=True):
        """FP32 PDEs: add each RK4 increment to the state with an exact two-sum
        and carry the rounding it lost into the next step (one more FP32 array),
        so long runs of small steps do not drift from FP64; getLocalSolution
        returns the state minus that correction (rbffd_pde_set_compensated_state)."""
        self.ctx.check(self.ctx.L.rbffd_pde_set_compensated_state(self.h, int(bool(on))), "set_compensated_state")

    TILE_STREAM_WEIGHTS, TILE_SLOT_SCHEDULE, TILE_PREFETCH, TILE_PIPELINE, TILE_DOUBLE_BUFFER = 1, 2, 4, 8, 16

    def setTiledShape(self, rows_per_block, lanes=1, stream_weights=False, slot_schedule=False, prefetch=False,
                      pipeline=False, double_buffer=False):
        """Tiled stage kernel of rows_per_block rows; stream_weights: bulk-copy
        weight streaming; slot_schedule: FP32 rows read their slots in the
        halo's conflict-avoiding order (4/8/16 tracers; every streamed
        operator in that order);
        prefetch: upcoming chunks of weights and indices asked of L2;
        pipeline: one operator streamed, the next chunks' weights and indices
        kept in flight in registers (combines with slot_schedule);
        double_buffer: one operator streamed by a persistent grid that copies
        the next tile's halo in while it computes the current one."""
        flags = ((self.TILE_STREAM_WEIGHTS if stream_weights else 0) | (self.TILE_SLOT_SCHEDULE if slot_schedule else 0) |
                 (self.TILE_PREFETCH if prefetch else 0) | (self.TILE_PIPELINE if pipeline else 0) |
                 (self.TILE_DOUBLE_BUFFER if double_buffer else 0))
        self.ctx.check(self.ctx.L.rbffd_pde_set_tiled_shape(self.h, rows_per_block, lanes, flags), "set_tiled_shape")

    def getTileFlags(self):
        """Flags of the tiled shape in use (TILE_* bits)."""
        f = ctypes.c_int()
        self.ctx.check(self.ctx.L.rbffd_pde_get_tile_flags(self.h, ctypes.byref(f)))
        return f.value

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.rbffd_pde_destroy(self.h)
            self.h = None


class CosineBell(TimeDependentPDE):
    """CosineBell(grid, der, earth_radius, velocity_angle, one_revolution_in_seconds, useHyperviscosity)
    (src/pdes/hyperbolic/cosine_bell.h:31-46)."""

    def __init__(self, grid, der, earth_radius, velocity_angle, one_revolution_in_seconds, useHyperviscosity,
                 dtype=F64, ntracers=1):
        u0 = (2.0 * np.pi * earth_radius) / one_revolution_in_seconds
        p = _lib.PdeParams(RHS_COSINE_BELL, ntracers, dtype, int(useHyperviscosity), earth_radius, velocity_angle, u0,
                           1.0, None, None)
        super().__init__(grid, der, p)


class HeatSphere(TimeDependentPDE):
    """u_t = kappa * Laplace-Beltrami(u) with the LSFC operator (rbffd.cpp:458-464)."""

    def __init__(self, grid, der, kappa=1.0, dtype=F64, ntracers=1):
        p = _lib.PdeParams(RHS_HEAT, ntracers, dtype, 0, 1.0, 0.0, 0.0, kappa, None, None)
        super().__init__(grid, der, p)


class Advection(TimeDependentPDE):
    """f = -(cu * D_lambda h + cv * D_theta h) [+ D_hv h] with caller-given per-node coefficients."""

    def __init__(self, grid, der, cu, cv, useHyperviscosity, dtype=F64, ntracers=1):
        """cv None: no D_theta term (f = -cu D_lambda h [+ D_hv h])."""
        self._cu, self._cv = _f64(cu), None if cv is None else _f64(cv)
        p = _lib.PdeParams(RHS_ADVECTION, ntracers, dtype, int(useHyperviscosity), 1.0, 0.0, 0.0, 1.0,
                           _dp(self._cu), _dp(self._cv))
        super().__init__(grid, der, p)


class VortexRollup(Advection):
    """VortexRollup (src/pdes/hyperbolic/vortex_rollup.h:7-30):
    f = -w(theta) * D_lambda h [+ D_hv h]; needs the LAMBDA (and HV) weights only."""

    def __init__(self, grid, der, useHyperviscosity, dtype=F64, ntracers=1):
        super().__init__(grid, der, vortex_rollup_coefficients(grid.nodes), None, useHyperviscosity, dtype=dtype,
                         ntracers=ntracers)


# ---------------------------------------------------------------------------
# serving

ERR_OOM, ERR_TIMEOUT, ERR_BUDGET, ERR_CANCELLED = -2, -4, -8, -10


def heat_params(kappa=1.0, dtype=F32):
    """Right-hand side of a served heat request (u_t = kappa * LSFC u)."""
    return _lib.PdeParams(RHS_HEAT, 1, dtype, 0, 1.0, 0.0, 0.0, kappa, None, None)


def cosine_bell_params(earth_radius, velocity_angle, one_revolution_in_seconds, useHyperviscosity, dtype=F32):
    """Right-hand side of a served solid-body advection request (CosineBell::solve)."""
    u0 = (2.0 * np.pi * earth_radius) / one_revolution_in_seconds
    return _lib.PdeParams(RHS_COSINE_BELL, 1, dtype, int(useHyperviscosity), earth_radius, velocity_angle, u0, 1.0,
                          None, None)


class Server:
    """Persistent request loop with continuous batching (rbffd_server_*).

    Requests (a grid with its weights, right-hand side parameters, an initial
    state, dt and a step count) are admitted against an HBM budget and advanced
    together, one launch per RK4 stage over all active requests."""

    ADMIT_ARRIVAL, ADMIT_SHORTEST = 0, 1

    def __init__(self, ctx, hbm_fraction=0.8, max_active=0, admission="arrival"):
        """admission: "arrival" (waiting requests admitted in arrival order) or
        "shortest" (least work first; rbffd_server_set_admission_order)."""
        if admission not in ("arrival", "shortest"):
            raise ValueError("admission must be 'arrival' or 'shortest'")
        self.ctx, self.L = ctx, ctx.L
        h = ctypes.c_void_p()
        ctx.check(self.L.rbffd_server_start(ctx.h, hbm_fraction, max_active, ctypes.byref(h)), "rbffd_server_start")
        self.h = h
        self._out = {}
        if admission != "arrival":
            self.setAdmissionOrder(admission)

    def setAdmissionOrder(self, admission):
        order = {"arrival": self.ADMIT_ARRIVAL, "shortest": self.ADMIT_SHORTEST}[admission]
        self.ctx.check(self.L.rbffd_server_set_admission_order(self.h, order), "rbffd_server_set_admission_order")

    def submit(self, grid, params, u0, dt, nsteps, cu=None, cv=None, out=None):
        """Queue a request; returns its id.  Raises RbffdError on a refused request.
        out: a float64 array of grid.N values that receives the result (by
        default a new one, returned by result())."""
        u = _f64(u0)
        assert u.shape == (grid.N,)
        if out is None:
            out = np.zeros(grid.N)
        assert out.dtype == np.float64 and out.shape == (grid.N,) and out.flags.c_contiguous
        keep = [u, out]
        if cu is not None:
            a, b = _f64(cu), _f64(cv)
            keep += [a, b]
            params = _lib.PdeParams(params.rhs_kind, params.ntracers, params.dtype, params.use_hv,
                                    params.sphere_radius, params.alpha, params.u0, params.kappa, _dp(a), _dp(b))
        req = _lib.Request(grid.h, params, _dp(u), dt, nsteps, _dp(out))
        rid = ctypes.c_uint64()
        self.ctx.check(self.L.rbffd_server_submit(self.h, ctypes.byref(req), ctypes.byref(rid)), "rbffd_server_submit")
        self._out[rid.value] = out
        return rid.value

    def poll(self, rid):
        """(done, status, latency_s, queue_s)."""
        d, s = ctypes.c_int(), ctypes.c_int()
        lat, q = ctypes.c_double(), ctypes.c_double()
        self.ctx.check(self.L.rbffd_server_poll(self.h, rid, ctypes.byref(d), ctypes.byref(s), ctypes.byref(lat),
                                                ctypes.byref(q)), "rbffd_server_poll")
        return bool(d.value), s.value, lat.value, q.value

    def wait(self, rid, timeout=600.0):
        """Status of the request once it is done (ERR_TIMEOUT if timeout passes first)."""
        return self.L.rbffd_server_wait(self.h, rid, timeout)

    def result(self, rid):
        """The request's result; raises unless it completed."""
        done, st, _, _ = self.poll(rid)
        if not done or st != 0:
            raise RbffdError(st if done else -6, "request %d has no result" % rid)
        return self._out[rid]

    def wait_idle(self, timeout=600.0):
        self.ctx.check(self.L.rbffd_server_wait_idle(self.h, timeout), "rbffd_server_wait_idle")

    def cancel(self, rid):
        self.ctx.check(self.L.rbffd_server_cancel(self.h, rid), "rbffd_server_cancel")

    def pause(self, paused=True):
        """Hold (or release) the stepping of admitted requests; admission continues."""
        self.ctx.check(self.L.rbffd_server_pause(self.h, int(paused)), "rbffd_server_pause")

    def inject_admission_failures(self, count):
        self.ctx.check(self.L.rbffd_server_inject_admission_failures(self.h, count))

    def stats(self):
        s = _lib.ServerStats()
        self.ctx.check(self.L.rbffd_server_get_stats(self.h, ctypes.byref(s)), "rbffd_server_get_stats")
        return {k: getattr(s, k) for k, _ in s._fields_}

    def stop(self):
        if getattr(self, "h", None):
            self.ctx.check(self.L.rbffd_server_stop(self.h), "rbffd_server_stop")
            self.h = None

    close = stop
