"""K3 parity: the fused RK4 stages against the oracle's restatement of
TimeDependentPDE::advanceRungeKutta4 (time_dependent_pde.cpp:172-304) with
CosineBell::solve (cosine_bell.cpp:23-70) and the heat right-hand side.

Weights are shared (the oracle's, installed with rbffd_weights_set) so the
comparison isolates the time stepping:
* FP64, one lane per stencil row: bit-exact after every tested step count
  (same accumulation order, same fused multiply-adds);
* FP64 with the autotuned shape (slots split across lanes): rel. L2 <= 1e-12;
* CUDA-graph replay and the unfused plain path: bit-exact with the fused path;
* FP32 (FP32 weights, state and accumulation): rel. L2 against the FP64 oracle
  <= 1e-5 on the tested horizons.
"""
import numpy as np
import pytest

import oracle as O
import rbffd_gpu_b200 as R
from tests.helpers import sphere_problem, cosine_bell_setup, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bell(ctx):
    N, n = 4096, 31
    xyz, st = sphere_problem(N, n, 1)
    types = O.LAMBDA | O.THETA | O.HV
    W = O.weights(xyz, st, None, 0.035 * np.sqrt(N), types, dim=2, poly_deg=2, hv_k=4, hv_scale=-1e-3 * N ** -4.0)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(types, grid, 2)
    for t, w in W.items():
        der.setWeights(t, w)
    p = cosine_bell_setup()
    cu, cv = O.cosine_bell_coeffs(xyz, a=p["a"], alpha=p["alpha"], u0=p["u0"])
    h0 = R.exact_cosine_bell(xyz)
    yield dict(xyz=xyz, st=st, W=W, grid=grid, der=der, p=p, cu=cu, cv=cv, h0=h0)
    grid.close()


def _oracle_bell(b, steps, u0=None):
    return O.rk4_advect(b["st"], None, b["W"][O.LAMBDA], b["W"][O.THETA], b["W"][O.HV], b["cu"], b["cv"],
                        b["h0"] if u0 is None else u0, b["p"]["dt"], steps)


def _gpu_bell(b, steps, dtype=R.F64, shape=(1, 256), graph=False, unfused=False):
    p = b["p"]
    pde = R.CosineBell(b["grid"], b["der"], p["a"], p["alpha"], p["T"], True, dtype=dtype)
    if shape is not None:
        pde.setShape(*shape)
    pde.fillInitialConditions(b["h0"])
    pde.advance(R.RK4, p["dt"], steps, graph=graph, unfused=unfused)
    out = pde.getLocalSolution()
    t = pde.getTime()
    pde.close()
    return out, t


@pytest.mark.parametrize("steps", [1, 4, 10])
def test_cosine_bell_fp64_bit_exact(bell, steps):
    out, t = _gpu_bell(bell, steps)
    assert np.array_equal(out, _oracle_bell(bell, steps))
    assert t == pytest.approx(steps * bell["p"]["dt"])


def test_cosine_bell_fp64_autotuned_shape(bell):
    out, _ = _gpu_bell(bell, 10, shape=None)
    assert rel_l2(out, _oracle_bell(bell, 10)) < 1e-12


@pytest.mark.parametrize("lanes", [2, 4, 8])
def test_cosine_bell_fp64_split_rows(bell, lanes):
    out, _ = _gpu_bell(bell, 10, shape=(lanes, 128))
    assert rel_l2(out, _oracle_bell(bell, 10)) < 1e-12


def _gpu_bell_tiled(b, steps, rows, lanes, dtype=R.F64, stream=False):
    p = b["p"]
    pde = R.CosineBell(b["grid"], b["der"], p["a"], p["alpha"], p["T"], True, dtype=dtype)
    pde.setTiledShape(rows, lanes, stream)
    assert pde.getShape()[2] == rows
    pde.fillInitialConditions(b["h0"])
    pde.advance(R.RK4, p["dt"], steps, graph=True)
    out = pde.getLocalSolution()
    pde.close()
    return out


@pytest.mark.parametrize("rows", [32, 64, 128, 256])
def test_cosine_bell_tiled_fp64_bit_exact(bell, rows):
    """Halo staged in shared memory, one lane per row: same arithmetic as the oracle."""
    assert np.array_equal(_gpu_bell_tiled(bell, 10, rows, 1), _oracle_bell(bell, 10))


@pytest.mark.parametrize("rows", [32, 64, 128])
def test_cosine_bell_streamed_weights_fp64_bit_exact(bell, rows):
    """Weights and indices streamed into shared memory by bulk copies (TMA)."""
    assert np.array_equal(_gpu_bell_tiled(bell, 10, rows, 1, stream=True), _oracle_bell(bell, 10))


def test_cosine_bell_streamed_weights_fp32(bell):
    assert rel_l2(_gpu_bell_tiled(bell, 10, 128, 1, dtype=R.F32, stream=True), _oracle_bell(bell, 10)) < 1e-5


@pytest.mark.parametrize("rows,lanes", [(64, 2), (128, 4)])
def test_cosine_bell_tiled_split_rows(bell, rows, lanes):
    assert rel_l2(_gpu_bell_tiled(bell, 10, rows, lanes), _oracle_bell(bell, 10)) < 1e-12


def test_graph_and_unfused_paths_bit_exact(bell):
    ref, _ = _gpu_bell(bell, 60)
    g, _ = _gpu_bell(bell, 60, graph=True)
    u, _ = _gpu_bell(bell, 60, unfused=True)
    assert np.array_equal(g, ref)
    assert np.array_equal(u, ref)


def test_cosine_bell_fp32_tolerance(bell):
    out, _ = _gpu_bell(bell, 10, dtype=R.F32, shape=None)
    assert rel_l2(out, _oracle_bell(bell, 10)) < 1e-5


@pytest.fixture(scope="module")
def heat(ctx):
    N, n = 10242, 50
    xyz, st = sphere_problem(N, n, 2)
    # eps h = 0.25 (the benchmark's rule; flatter choices make kappa ~ 1e15 at large N)
    W = O.weights(xyz, st, None, 0.25 / np.sqrt(4 * np.pi / N), O.LSFC, dim=2, poly_deg=3)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(O.LSFC, grid, 2)
    der.setWeights(O.LSFC, W[O.LSFC])
    lmax = 20
    c = np.random.default_rng(2).standard_normal((lmax + 1) ** 2)
    u0 = R.exact_sph_heat(xyz, lmax, c, 0.0)
    yield dict(xyz=xyz, st=st, W=W, grid=grid, der=der, u0=u0, c=c, lmax=lmax)
    grid.close()


def _gpu_heat(h, steps, dt, dtype=R.F64, shape=(1, 256), graph=False):
    pde = R.HeatSphere(h["grid"], h["der"], 1.0, dtype=dtype)
    if shape is not None:
        pde.setShape(*shape)
    pde.fillInitialConditions(h["u0"])
    pde.advance(R.RK4, dt, steps, graph=graph)
    out = pde.getLocalSolution()
    pde.close()
    return out


def test_heat_fp64_bit_exact(heat):
    out = _gpu_heat(heat, 25, 1e-6)
    assert np.array_equal(out, O.rk4_heat(heat["st"], None, heat["W"][O.LSFC], heat["u0"], 1e-6, 25))


def test_heat_fp32_tolerance_and_exact_decay(heat):
    steps, dt = 100, 1e-6
    ref = O.rk4_heat(heat["st"], None, heat["W"][O.LSFC], heat["u0"], dt, steps)
    out = _gpu_heat(heat, steps, dt, dtype=R.F32, shape=None, graph=True)
    assert rel_l2(out, ref) < 1e-5
    ex = R.exact_sph_heat(heat["xyz"], heat["lmax"], heat["c"], steps * dt)
    assert rel_l2(ref, ex) < 1e-3


@pytest.mark.parametrize("dtype,tol,tiled", [(R.F64, 0.0, None), (R.F32, 1e-5, None), (R.F64, 0.0, (64, 1)),
                                             (R.F64, 1e-12, (32, 4)), (R.F32, 1e-5, (128, 2)),
                                             (R.F64, 0.0, (64, 1, True)), (R.F32, 1e-5, (128, 1, True)),
                                             (R.F64, 0.0, (64, 1, False, False, True)),
                                             (R.F32, 1e-5, (128, 1, False, False, True))])
def test_multi_tracer_advection(bell, dtype, tol, tiled):
    T = 16
    rng = np.random.default_rng(4)
    xyz = bell["xyz"]
    cen = rng.normal(size=(T, 3))
    cen /= np.linalg.norm(cen, axis=1)[:, None]
    u0 = np.exp(-8.0 * ((xyz[:, None, :] - cen[None, :, :]) ** 2).sum(2))  # Gaussian hills, [N][T]
    steps, dt = 10, bell["p"]["dt"]
    ref = O.rk4_advect(bell["st"], None, bell["W"][O.LAMBDA], bell["W"][O.THETA], bell["W"][O.HV], bell["cu"],
                       bell["cv"], u0, dt, steps)
    pde = R.Advection(bell["grid"], bell["der"], bell["cu"], bell["cv"], True, dtype=dtype, ntracers=T)
    if tiled:
        pde.setTiledShape(*tiled)
    elif tol == 0.0:
        pde.setShape(1, 256)  # one lane per (row, tracer group): the oracle's summation order
    pde.fillInitialConditions(u0)
    pde.advance(R.RK4, dt, steps, graph=True)
    out = pde.getLocalSolution()
    pde.close()
    if tol == 0.0:
        assert np.array_equal(out, ref)
    else:
        assert rel_l2(out, ref) < tol


@pytest.mark.parametrize("ntr,shape", [(1, None), (1, (128, 1)), (16, None), (16, (128, 1)), (16, (64, 1, True))])
def test_fused_advection_operator_fp32(bell, ntr, shape):
    """FP32 advection with the three operators fused into one
    (-(cu Wl + cv Wt) + Whv, formed in FP64, rounded once): within 1e-5
    (rel. L2) of the FP64 oracle's three-operator RK4; switching back gives the
    three-operator FP32 bits again."""
    p = bell["p"]
    rng = np.random.default_rng(12)
    u0 = bell["h0"] if ntr == 1 else rng.random((bell["xyz"].shape[0], ntr))
    steps, dt = 10, p["dt"]
    ref = O.rk4_advect(bell["st"], None, bell["W"][O.LAMBDA], bell["W"][O.THETA], bell["W"][O.HV], bell["cu"],
                       bell["cv"], u0, dt, steps)

    def run(fused_then_off=False, fused=True):
        pde = R.Advection(bell["grid"], bell["der"], bell["cu"], bell["cv"], True, dtype=R.F32, ntracers=ntr)
        if shape is not None:
            pde.setTiledShape(*shape)
        else:
            pde.setShape(1, 256)
        if fused or fused_then_off:
            pde.setFusedOperator(True)
        pde.fillInitialConditions(u0)
        if fused_then_off:
            pde.advance(R.RK4, dt, 30, graph=True)  # a graph of the fused stages exists now
            pde.setFusedOperator(False)
            pde.fillInitialConditions(u0)
            pde.setTime(0.0)
        pde.advance(R.RK4, dt, steps, graph=True)
        out = pde.getLocalSolution()
        pde.close()
        return out

    fused = run()
    assert rel_l2(fused, ref) < 1e-5
    assert np.array_equal(run(fused_then_off=True, fused=False), run(fused=False))


@pytest.mark.parametrize("ntr", [1, 16])
def test_fused_operator_fp64(bell, ntr):
    """FP64 advection on its fused operator (formed in FP64, one weight array
    per stage): within FP64 rounding of the three-operator path (itself within
    rounding of the oracle)."""
    rng = np.random.default_rng(80 + ntr)
    u0 = bell["h0"] if ntr == 1 else bell["h0"][:, None] * (1.0 + 0.1 * rng.random((1, ntr)))
    steps = 20

    def run(fused):
        pde = R.Advection(bell["grid"], bell["der"], bell["cu"], bell["cv"], True, dtype=R.F64, ntracers=ntr)
        if fused:
            pde.setFusedOperator(True)
        pde.fillInitialConditions(u0)
        pde.advance(R.RK4, bell["p"]["dt"], steps, graph=True)
        out = pde.getLocalSolution()
        pde.close()
        return out

    three = run(False)
    assert rel_l2(run(True), three) <= 1e-12
    if ntr == 1:
        assert rel_l2(three, _oracle_bell(bell, steps)) <= 1e-14


def test_fused_operator_errors(bell, heat):
    """The reference's (unfused) arithmetic keeps the three operators either
    way round; heat has no operator to fuse."""
    pde = R.CosineBell(bell["grid"], bell["der"], bell["p"]["a"], bell["p"]["alpha"], bell["p"]["T"], True,
                       dtype=R.F64)
    pde.setArithmetic(R.ARITH_UNFUSED)
    with pytest.raises(R.RbffdError) as e:
        pde.setFusedOperator(True)
    assert e.value.status == -5
    pde.setFusedOperator(False)  # off is always accepted
    pde.setArithmetic(R.ARITH_FUSED)
    pde.setFusedOperator(True)
    with pytest.raises(R.RbffdError) as e:
        pde.setArithmetic(R.ARITH_UNFUSED)
    assert e.value.status == -5
    pde.close()
    hp = R.HeatSphere(heat["grid"], heat["der"], 1.0, dtype=R.F32)
    with pytest.raises(R.RbffdError) as e:
        hp.setFusedOperator(True)
    assert e.value.status == -5
    hp.close()


@pytest.mark.parametrize("dtype", [R.F64, R.F32])
def test_autotuner_leaves_the_state_untouched(heat, dtype):
    """The autotuner times full RK4 steps on the PDE's own buffers (dt = 0,
    the state saved and restored): a PDE tuned on its first advance gives the
    same bits as one forced to the chosen shape from the start."""
    ctx2 = R.Context(0)  # a fresh context: no tuned shape cached yet
    grid = R.Grid(ctx2, heat["xyz"], heat["st"])
    der = R.RBFFD(R.LSFC, grid, 2)
    der.setWeights(R.LSFC, heat["W"][O.LSFC])
    tuned = R.HeatSphere(grid, der, 1.0, dtype=dtype)
    tuned.fillInitialConditions(heat["u0"])
    tuned.advance(R.RK4, 1e-6, 7)
    lanes, block, rows = tuned.getShape()
    flags = tuned.getTileFlags()
    out_tuned = tuned.getLocalSolution()
    tuned.close()
    forced = R.HeatSphere(grid, der, 1.0, dtype=dtype)
    if rows > 0:
        forced.setTiledShape(rows, lanes, stream_weights=bool(flags & 1), slot_schedule=bool(flags & 2),
                             prefetch=bool(flags & 4))
    else:
        forced.setShape(lanes, block)
    forced.fillInitialConditions(heat["u0"])
    forced.advance(R.RK4, 1e-6, 7)
    assert np.array_equal(forced.getLocalSolution(), out_tuned)
    forced.close()
    grid.close()
    ctx2.close()


@pytest.mark.parametrize("ntr", [4, 8, 16])
def test_slot_schedule_heat_multi_tracer(heat, ntr):
    """FP32 heat with 4, 8 or 16 tracers, rows reading their slots in the
    halo's conflict-avoiding order: within FP32 rounding of the same tile in
    stencil order, and within 1e-5 of the FP64 oracle."""
    rng = np.random.default_rng(30 + ntr)
    u0 = heat["u0"][:, None] * (1.0 + 0.1 * rng.random((1, ntr)))
    steps, dt = 40, 1e-6
    ref = O.rk4_heat(heat["st"], None, heat["W"][O.LSFC], u0, dt, steps)

    def run(sched):
        pde = R.HeatSphere(heat["grid"], heat["der"], 1.0, dtype=R.F32, ntracers=ntr)
        pde.setTiledShape(128, 1, slot_schedule=sched)
        assert pde.getTileFlags() == (R.TimeDependentPDE.TILE_SLOT_SCHEDULE if sched else 0)
        pde.fillInitialConditions(u0)
        pde.advance(R.RK4, dt, steps, graph=True)
        out = pde.getLocalSolution()
        pde.close()
        return out

    s, plain = run(True), run(False)
    assert rel_l2(s, ref) < 1e-5
    assert rel_l2(s, plain) < 2e-6
    assert not np.array_equal(s, plain)  # a different summation order


def test_slot_schedule_fused_advection_and_refresh(bell):
    """16 tracers with the fused advection operator in slot order: within 1e-5
    of the FP64 oracle; after the operator is fused again (off, on) the
    scheduled copy follows it (same bits as a fresh PDE)."""
    T = 16
    rng = np.random.default_rng(31)
    u0 = rng.random((bell["xyz"].shape[0], T))
    steps, dt = 10, bell["p"]["dt"]
    ref = O.rk4_advect(bell["st"], None, bell["W"][O.LAMBDA], bell["W"][O.THETA], bell["W"][O.HV], bell["cu"],
                       bell["cv"], u0, dt, steps)

    def make():
        pde = R.Advection(bell["grid"], bell["der"], bell["cu"], bell["cv"], True, dtype=R.F32, ntracers=T)
        pde.setFusedOperator(True)
        pde.setTiledShape(128, 1, slot_schedule=True)
        pde.fillInitialConditions(u0)
        return pde

    pde = make()
    pde.advance(R.RK4, dt, steps, graph=True)
    first = pde.getLocalSolution()
    assert rel_l2(first, ref) < 1e-5
    pde.setFusedOperator(False)
    pde.setFusedOperator(True)
    pde.fillInitialConditions(u0)
    pde.setTime(0.0)
    pde.advance(R.RK4, dt, steps, graph=True)
    assert np.array_equal(pde.getLocalSolution(), first)
    pde.close()


@pytest.mark.parametrize("ntr", [4, 16])
def test_slot_schedule_three_operator_advection(bell, ntr):
    """FP32 advection streaming its three operators (d/dlambda, d/dtheta,
    hyperviscosity), all in the halo's slot order: within 1e-5 of the FP64
    oracle and within FP32 rounding of stencil order."""
    rng = np.random.default_rng(40 + ntr)
    u0 = rng.random((bell["xyz"].shape[0], ntr))
    steps, dt = 10, bell["p"]["dt"]
    ref = O.rk4_advect(bell["st"], None, bell["W"][O.LAMBDA], bell["W"][O.THETA], bell["W"][O.HV], bell["cu"],
                       bell["cv"], u0, dt, steps)

    def run(sched):
        pde = R.Advection(bell["grid"], bell["der"], bell["cu"], bell["cv"], True, dtype=R.F32, ntracers=ntr)
        pde.setTiledShape(128, 1, slot_schedule=sched)
        assert pde.getTileFlags() == (R.TimeDependentPDE.TILE_SLOT_SCHEDULE if sched else 0)
        pde.fillInitialConditions(u0)
        pde.advance(R.RK4, dt, steps, graph=True)
        out = pde.getLocalSolution()
        pde.close()
        return out

    s, plain = run(True), run(False)
    assert rel_l2(s, ref) < 1e-5
    assert rel_l2(s, plain) < 2e-6
    assert not np.array_equal(s, plain)


def test_slot_schedule_follows_changed_weights(ctx):
    """The scheduled copies follow the grid's operators: after one operator's
    weights change, a PDE that ran before gives a fresh PDE's bits."""
    N, n, T = 2562, 31, 8
    xyz, st = sphere_problem(N, n, 5)
    W = O.weights(xyz, st, None, 6.0, O.LAMBDA | O.THETA | O.HV, dim=2, poly_deg=2, hv_k=4,
                  hv_scale=-1e-3 * N ** -4.0)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(R.LAMBDA | R.THETA | R.HV, grid, 2)
    for t, w in W.items():
        der.setWeights(t, w)
    rng = np.random.default_rng(41)
    cu, cv, u0 = rng.standard_normal(N), rng.standard_normal(N), rng.random((N, T))

    def make():
        pde = R.Advection(grid, der, cu, cv, True, dtype=R.F32, ntracers=T)
        pde.setTiledShape(128, 1, slot_schedule=True)
        pde.fillInitialConditions(u0)
        return pde

    old = make()
    old.advance(R.RK4, 1e-3, 5, graph=True)
    der.setWeights(R.HV, 3.0 * W[O.HV])
    old.fillInitialConditions(u0)
    old.setTime(0.0)
    old.advance(R.RK4, 1e-3, 5, graph=True)
    new = make()
    new.advance(R.RK4, 1e-3, 5, graph=True)
    assert np.array_equal(old.getLocalSolution(), new.getLocalSolution())
    old.close()
    new.close()
    grid.close()


def test_slot_schedule_refused_where_it_does_not_apply(bell, heat):
    cases = [R.HeatSphere(heat["grid"], heat["der"], 1.0, dtype=R.F64, ntracers=4),   # FP64
             R.HeatSphere(heat["grid"], heat["der"], 1.0, dtype=R.F32, ntracers=1),   # scalar records
             R.HeatSphere(heat["grid"], heat["der"], 1.0, dtype=R.F32, ntracers=32)]  # 128-byte records
    for pde in cases:
        with pytest.raises(R.RbffdError) as e:
            pde.setTiledShape(128, 1, slot_schedule=True)
        assert e.value.status == -5
        pde.close()
    pde = R.HeatSphere(heat["grid"], heat["der"], 1.0, dtype=R.F32, ntracers=4)
    with pytest.raises(R.RbffdError) as e:
        pde.setTiledShape(128, 2, slot_schedule=True)  # one lane per row only
    assert e.value.status == -1
    with pytest.raises(R.RbffdError) as e:
        pde.setTiledShape(128, 1, stream_weights=True, slot_schedule=True)
    assert e.value.status == -1
    pde.close()


@pytest.mark.slow
def test_heat_benchmark_grid_parity(ctx):
    """The benchmark's own heat configuration: N = 163842, n = 50, degree 3,
    eps h = 0.25, the whole 500-step workload.  FP64 with one lane per row
    equals the oracle bit for bit; FP64 with the autotuned shape within 1e-12;
    FP32 (autotuned) within 1e-5 of the FP64 oracle (rel. L2)."""
    N, n, steps, dt = 163842, 50, 500, 1e-6
    xyz = R.fibonacci_nodes(N, 2)
    st = R.knn_stencils(xyz, n)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(R.LSFC, grid, 2)
    der.setEpsilon(0.25 / np.sqrt(4 * np.pi / N))
    der.setPolynomialDegree(3)
    der.computeAllWeightsForAllStencils()
    W = der.getWeights(R.LSFC)
    u0 = R.exact_sph_heat(xyz, 20, np.random.default_rng(2).standard_normal(441), 0.0)
    ref = O.rk4_heat(st, None, W, u0, dt, steps, nthreads=O.max_threads())
    h = dict(grid=grid, der=der, u0=u0)
    assert np.array_equal(_gpu_heat(h, steps, dt, shape=(1, 256), graph=True), ref)
    assert rel_l2(_gpu_heat(h, steps, dt, shape=None, graph=True), ref) <= 1e-12
    assert rel_l2(_gpu_heat(h, steps, dt, dtype=R.F32, shape=None, graph=True), ref) <= 1e-5
    grid.close()


@pytest.mark.parametrize("dtype,ntr", [(R.F64, 1), (R.F64, 8), (R.F64, 16), (R.F32, 1), (R.F32, 4), (R.F32, 16)])
def test_register_pipelined_tile_heat(heat, dtype, ntr):
    """The tiled kernel with the weight and index stream pipelined in
    registers (RBFFD_TILE_PIPELINE): the same bits as the plain tiled kernel
    with one lane group per row, for every node width it serves; FP64 equals
    the oracle bit for bit."""
    rng = np.random.default_rng(40 + ntr)
    u0 = heat["u0"] if ntr == 1 else heat["u0"][:, None] * (1.0 + 0.1 * rng.random((1, ntr)))
    steps, dt = 30, 1e-6

    def run(pipe, rows=128):
        pde = R.HeatSphere(heat["grid"], heat["der"], 1.0, dtype=dtype, ntracers=ntr)
        pde.setTiledShape(rows, 1, pipeline=pipe)
        assert pde.getTileFlags() == (R.TimeDependentPDE.TILE_PIPELINE if pipe else 0)
        pde.fillInitialConditions(u0)
        pde.advance(R.RK4, dt, steps, graph=True)
        out = pde.getLocalSolution()
        pde.close()
        return out

    piped = run(True)
    assert np.array_equal(piped, run(False))
    assert np.array_equal(run(True, 64), piped)
    if dtype == R.F64:
        assert np.array_equal(piped, O.rk4_heat(heat["st"], None, heat["W"][O.LSFC], u0, dt, steps))


@pytest.mark.parametrize("dtype,ntr", [(R.F64, 1), (R.F64, 2), (R.F64, 4), (R.F64, 16), (R.F32, 1), (R.F32, 8),
                                       (R.F32, 16)])
def test_double_buffered_tile_heat(heat, dtype, ntr):
    """The persistent tiled kernel that copies the next tile's halo in while
    it computes the current one (RBFFD_TILE_DOUBLE_BUFFER): the same bits as
    the plain tiled kernel for every node width it serves; FP64 equals the
    oracle bit for bit; it combines with no other tiled-shape flag."""
    rng = np.random.default_rng(60 + ntr)
    u0 = heat["u0"] if ntr == 1 else heat["u0"][:, None] * (1.0 + 0.1 * rng.random((1, ntr)))
    steps, dt = 30, 1e-6

    def run(db, rows=128):
        pde = R.HeatSphere(heat["grid"], heat["der"], 1.0, dtype=dtype, ntracers=ntr)
        pde.setTiledShape(rows, 1, double_buffer=db)
        assert pde.getTileFlags() == (R.TimeDependentPDE.TILE_DOUBLE_BUFFER if db else 0)
        pde.fillInitialConditions(u0)
        pde.advance(R.RK4, dt, steps, graph=True)
        out = pde.getLocalSolution()
        pde.close()
        return out

    db = run(True)
    assert np.array_equal(db, run(False))
    assert np.array_equal(run(True, 64), db)
    if dtype == R.F64:
        assert np.array_equal(db, O.rk4_heat(heat["st"], None, heat["W"][O.LSFC], u0, dt, steps))
    pde = R.HeatSphere(heat["grid"], heat["der"], 1.0, dtype=dtype, ntracers=ntr)
    with pytest.raises(R.RbffdError):
        pde.setTiledShape(128, 1, pipeline=True, double_buffer=True)
    with pytest.raises(R.RbffdError):
        pde.setTiledShape(128, 2, double_buffer=True)
    pde.close()


@pytest.mark.parametrize("dtype,ntr", [(R.F64, 16), (R.F32, 32)])
def test_double_buffered_tile_walks_several_tiles_per_block(ctx, dtype, ntr):
    """A grid of 40962 nodes in 64-row tiles with 16 (FP64) / 32 (FP32) values
    per node has more tiles than the persistent grid has blocks, so each block
    walks several tiles through both halo buffers: the same bits as the plain
    tiled kernel and the register-pipelined one, with and without a graph."""
    N, n = 40962, 50
    xyz = R.fibonacci_nodes(N, 2)
    st = R.knn_stencils(xyz, n)
    grid = R.Grid(ctx, xyz, st)
    der = R.RBFFD(R.LSFC, grid, 2)
    der.setEpsilon(0.25 / np.sqrt(4 * np.pi / N))
    der.setPolynomialDegree(3)
    der.computeAllWeightsForAllStencils()
    rng = np.random.default_rng(9)
    u0 = R.exact_sph_heat(xyz, 12, rng.standard_normal(169), 0.0)[:, None] * (1.0 + 0.1 * rng.random((1, ntr)))
    steps, dt = 12, 1e-7

    def run(graph, **flags):
        pde = R.HeatSphere(grid, der, 1.0, dtype=dtype, ntracers=ntr)
        pde.setTiledShape(64, 1, **flags)
        pde.fillInitialConditions(u0)
        pde.advance(R.RK4, dt, steps, graph=graph)
        out = pde.getLocalSolution()
        pde.close()
        return out

    db = run(True, double_buffer=True)
    assert np.isfinite(db).all()
    assert np.array_equal(db, run(True))
    assert np.array_equal(db, run(True, pipeline=True))
    assert np.array_equal(db, run(False, double_buffer=True))
    grid.close()


def test_double_buffered_tile_fused_advection(bell):
    """16-tracer FP32 advection on its fused operator: the double-buffered
    persistent kernel gives the plain tiled kernel's bits; a three-operator
    PDE refuses it."""
    T = 16
    rng = np.random.default_rng(18)
    cen = rng.normal(size=(T, 3))
    cen /= np.linalg.norm(cen, axis=1)[:, None]
    u0 = np.exp(-8.0 * ((bell["xyz"][:, None, :] - cen[None, :, :]) ** 2).sum(2))
    outs = []
    for db in (True, False):
        pde = R.Advection(bell["grid"], bell["der"], bell["cu"], bell["cv"], True, dtype=R.F32, ntracers=T)
        pde.setFusedOperator(True)
        pde.setTiledShape(128, 1, double_buffer=db)
        pde.fillInitialConditions(u0)
        pde.advance(R.RK4, bell["p"]["dt"], 10, graph=True)
        outs.append(pde.getLocalSolution())
        pde.close()
    assert np.array_equal(outs[0], outs[1])
    p3 = R.Advection(bell["grid"], bell["der"], bell["cu"], bell["cv"], True, dtype=R.F32, ntracers=T)
    with pytest.raises(R.RbffdError):
        p3.setTiledShape(128, 1, double_buffer=True)
    p3.close()


def test_register_pipelined_tile_fused_advection_with_schedule(bell):
    """16-tracer FP32 advection on its fused operator, rows in the slot
    schedule: the pipelined kernel gives the plain scheduled kernel's bits; a
    three-operator PDE refuses the pipeline."""
    T = 16
    rng = np.random.default_rng(8)
    cen = rng.normal(size=(T, 3))
    cen /= np.linalg.norm(cen, axis=1)[:, None]
    u0 = np.exp(-8.0 * ((bell["xyz"][:, None, :] - cen[None, :, :]) ** 2).sum(2))
    outs = []
    for pipe in (True, False):
        pde = R.Advection(bell["grid"], bell["der"], bell["cu"], bell["cv"], True, dtype=R.F32, ntracers=T)
        pde.setFusedOperator(True)
        pde.setTiledShape(128, 1, slot_schedule=True, pipeline=pipe)
        pde.fillInitialConditions(u0)
        pde.advance(R.RK4, bell["p"]["dt"], 10, graph=True)
        outs.append(pde.getLocalSolution())
        pde.close()
    assert np.array_equal(outs[0], outs[1])
    p3 = R.Advection(bell["grid"], bell["der"], bell["cu"], bell["cv"], True, dtype=R.F32, ntracers=T)
    with pytest.raises(R.RbffdError):
        p3.setTiledShape(128, 1, pipeline=True)
    p3.close()
