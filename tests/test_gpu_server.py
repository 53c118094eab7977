"""Serving: the persistent request loop with continuous batching (rbffd_server_*).

* FP64 served requests equal the oracle's RK4 (TimeDependentPDE::advanceRungeKutta4,
  time_dependent_pde.cpp:172-304) bit for bit, heat and cosine bell;
* every request's result is identical alone and in a mix of grids, stencil
  sizes, right-hand sides, dtypes and step counts with staggered arrivals;
  FP32 heat results are within FP32 rounding of the one-lane rbffd_pde_advance
  result, FP32 advection (one fused operator per bank) is within 1e-5 of the
  FP64 oracle; FP32 banks keep a compensated state, so long runs of small
  steps stay close to FP64;
* admission: a request that can never fit the HBM budget is refused at
  submission; a budget with room for one request runs them one at a time;
* cancellation (pending and active), injected admission failures, malformed
  requests and zero-step requests.
"""
import time

import numpy as np
import pytest

import oracle as O
import rbffd_gpu_b200 as R
from tests.helpers import sphere_problem, cosine_bell_setup, rel_l2

pytestmark = pytest.mark.gpu


def _grid(ctx, N, n, seed):
    xyz, st = sphere_problem(N, n, seed)
    h = np.sqrt(4 * np.pi / N)
    W = O.weights(xyz, st, None, 0.25 / h, O.LSFC, dim=2, poly_deg=3)
    W.update(O.weights(xyz, st, None, 0.035 * np.sqrt(N), O.LAMBDA | O.THETA | O.HV, dim=2, poly_deg=2, hv_k=4,
                       hv_scale=-1e-3 * N ** -4.0))
    g = R.Grid(ctx, xyz, st)
    der = R.RBFFD(O.LSFC | O.LAMBDA | O.THETA | O.HV, g, 2)
    for t, w in W.items():
        der.setWeights(t, w)
    return dict(xyz=xyz, st=st, W=W, grid=g, der=der, N=N)


@pytest.fixture(scope="module")
def grids(ctx):
    gs = [_grid(ctx, 2562, 31, 5), _grid(ctx, 4096, 50, 6)]
    yield gs
    for g in gs:
        g["grid"].close()


def _heat_u0(g, seed):
    c = np.random.default_rng(seed).standard_normal(11 ** 2)
    return R.exact_sph_heat(g["xyz"], 10, c, 0.0)


def _bell_u0(g, seed):
    rng = np.random.default_rng(seed)
    cen = rng.normal(size=3)
    cen /= np.linalg.norm(cen)
    return np.exp(-6.0 * ((g["xyz"] - cen) ** 2).sum(1))


BELL = cosine_bell_setup()


def _bell_params(dtype):
    return R.cosine_bell_params(BELL["a"], BELL["alpha"], BELL["T"], True, dtype=dtype)


def _specs(grids):
    """A mix: both grids, heat and advection, FP32 and FP64, 7 to 90 steps."""
    out = []
    for k in range(10):
        g = grids[k % 2]
        dtype = R.F32 if k % 3 else R.F64
        steps = [7, 90, 23, 41, 12, 66, 30, 9, 55, 18][k]
        if k % 4 < 2:
            out.append((g, R.heat_params(1.0 + 0.1 * k, dtype), _heat_u0(g, k), 1e-5, steps))
        else:
            out.append((g, _bell_params(dtype), _bell_u0(g, k), BELL["dt"], steps))
    return out


def _submit(srv, spec):
    g, p, u0, dt, steps = spec
    return srv.submit(g["grid"], p, u0, dt, steps)


def test_served_fp64_matches_oracle_bit_exact(ctx, grids):
    g0, g1 = grids
    srv = R.Server(ctx)
    try:
        u_h = _heat_u0(g0, 1)
        u_b = _bell_u0(g1, 2)
        rh = srv.submit(g0["grid"], R.heat_params(1.0, R.F64), u_h, 1e-5, 12)
        rb = srv.submit(g1["grid"], _bell_params(R.F64), u_b, BELL["dt"], 9)
        assert srv.wait(rh) == 0 and srv.wait(rb) == 0
        ref_h = O.rk4_heat(g0["st"], None, g0["W"][O.LSFC], u_h, 1e-5, 12)
        assert np.array_equal(srv.result(rh), ref_h)
        cu, cv = O.cosine_bell_coeffs(g1["xyz"], a=BELL["a"], alpha=BELL["alpha"], u0=BELL["u0"])
        ref_b = O.rk4_advect(g1["st"], None, g1["W"][O.LAMBDA], g1["W"][O.THETA], g1["W"][O.HV], cu, cv, u_b,
                             BELL["dt"], 9)
        assert np.array_equal(srv.result(rb), ref_b)
    finally:
        srv.stop()


def test_alone_and_in_mix_identical(ctx, grids):
    specs = _specs(grids)
    srv = R.Server(ctx)
    try:
        alone = []
        for s in specs:
            rid = _submit(srv, s)
            assert srv.wait(rid) == 0
            alone.append(srv.result(rid).copy())
        st0 = srv.stats()
        # the mix: half now, the rest once the first batch runs (they join at a step boundary)
        ids = [_submit(srv, s) for s in specs[:5]]
        t0 = time.time()
        while srv.poll(ids[1])[3] < 0 and time.time() - t0 < 10:
            time.sleep(0.001)
        ids += [_submit(srv, s) for s in specs[5:]]
        srv.wait_idle(120)
        for k, (a, rid) in enumerate(zip(alone, ids)):
            done, status, lat, q = srv.poll(rid)
            assert done and status == 0, (k, status)
            assert lat >= q >= 0
            assert np.array_equal(srv.result(rid), a), k
        st = srv.stats()
        assert st["max_active_seen"] >= 2
        assert st["completed"] == 20 and st["failed"] == 0
        assert st["slots_reused"] > st0["slots_reused"]  # finished requests' buffers serve later ones
        assert st["node_updates"] == pytest.approx(2 * sum(s[0]["N"] * s[4] for s in specs))
    finally:
        srv.stop()


def test_many_requests_on_one_grid_share_launches_bit_exact(ctx, grids):
    """11 FP64 requests on one grid: groups of up to 8 read the operators once
    per row for all members; each member still equals the oracle bit for bit."""
    g = grids[0]
    srv = R.Server(ctx)
    try:
        specs = [(_heat_u0(g, 20 + k), 1.0 + 0.05 * k, 5 + 3 * k) for k in range(11)]
        srv.pause()  # all 11 are admitted before the first batch: one group of 8 and one of 3
        ids = [srv.submit(g["grid"], R.heat_params(kap, R.F64), u, 1e-5, steps) for u, kap, steps in specs]
        t0 = time.time()
        while any(srv.poll(i)[3] < 0 for i in ids) and time.time() - t0 < 30:
            time.sleep(0.001)
        assert srv.stats()["ticks"] == 0
        srv.pause(False)
        srv.wait_idle(60)
        for (u, kap, steps), rid in zip(specs, ids):
            ref = O.rk4_heat(g["st"], None, g["W"][O.LSFC], u, 1e-5, steps, kappa=kap)
            assert np.array_equal(srv.result(rid), ref), (kap, steps)
        assert srv.stats()["max_active_seen"] == 11
    finally:
        srv.stop()


def test_served_fp32_heat_against_oracle_and_pde_path(ctx, grids):
    """FP32 banks sum each row in the halo's conflict-avoiding slot order:
    within FP32 rounding of the one-lane FP32 PDE path (stencil order) and
    within 1e-5 of the FP64 oracle."""
    g = grids[1]
    u0 = _heat_u0(g, 3)
    srv = R.Server(ctx)
    try:
        rid = srv.submit(g["grid"], R.heat_params(1.0, R.F32), u0, 1e-5, 40)
        assert srv.wait(rid) == 0
        served = srv.result(rid)
    finally:
        srv.stop()
    pde = R.HeatSphere(g["grid"], g["der"], 1.0, dtype=R.F32)
    pde.setShape(1, 128)
    pde.fillInitialConditions(u0)
    pde.advance(R.RK4, 1e-5, 40)
    ref32 = pde.getLocalSolution()
    pde.close()
    ref = O.rk4_heat(g["st"], None, g["W"][O.LSFC], u0, 1e-5, 40)
    assert rel_l2(served, ref32) < 2e-6
    assert rel_l2(served, ref) < 1e-5
    assert not np.array_equal(served, ref32)  # the scheduled order is in use


def test_served_fp32_long_heat_keeps_its_small_increments(ctx, grids):
    """2000 small heat steps (each moves the state by about 1e-4 of itself):
    rounding u + increment to FP32 every step loses most of the increment's
    bits, and the FP32 PDE path drifts by 1.6e-6 from the FP64 result; the
    FP32 banks carry each step's lost part into the next (compensated sum)
    and stay within 2e-7 of it, 40x closer."""
    g = grids[1]
    u0 = _heat_u0(g, 3)
    dt, steps = 1e-6, 2000

    def pde_run(dtype):
        pde = R.HeatSphere(g["grid"], g["der"], 1.0, dtype=dtype)
        pde.setShape(1, 128)
        pde.fillInitialConditions(u0)
        pde.advance(R.RK4, dt, steps, graph=True)
        out = pde.getLocalSolution()
        pde.close()
        return out

    ref, plain32 = pde_run(R.F64), pde_run(R.F32)
    srv = R.Server(ctx)
    try:
        rid = srv.submit(g["grid"], R.heat_params(1.0, R.F32), u0, dt, steps)
        assert srv.wait(rid) == 0
        served = srv.result(rid)
    finally:
        srv.stop()
    assert rel_l2(served, ref) < 2e-7
    assert rel_l2(plain32, ref) > 5 * rel_l2(served, ref)


def test_served_fp32_advection_fused_operator(ctx, grids):
    """FP32 advection banks apply one fused operator per bank,
    Wf = -(cu W_lambda + cv W_theta) + W_hv formed in FP64 and rounded once to
    FP32: within 1e-5 relative L2 of the FP64 oracle after 30 steps, and
    identical whether the request runs alone or beside others in its bank.
    (dt/20: these weights, eps = 0.035 sqrt(N), carry growing modes that
    amplify any rounding difference over full cosine-bell steps.)"""
    g = grids[1]
    dt = BELL["dt"] / 20
    u_b = [_bell_u0(g, 30 + k) for k in range(3)]
    srv = R.Server(ctx)
    try:
        alone = srv.submit(g["grid"], _bell_params(R.F32), u_b[0], dt, 30)
        assert srv.wait(alone) == 0
        srv.pause()
        ids = [srv.submit(g["grid"], _bell_params(R.F32), u, dt, 30) for u in u_b]
        while any(srv.poll(i)[3] < 0 for i in ids):
            time.sleep(0.001)
        srv.pause(False)
        srv.wait_idle(60)
        assert np.array_equal(srv.result(ids[0]), srv.result(alone))
        cu, cv = O.cosine_bell_coeffs(g["xyz"], a=BELL["a"], alpha=BELL["alpha"], u0=BELL["u0"])
        for u, rid in zip(u_b, ids):
            ref = O.rk4_advect(g["st"], None, g["W"][O.LAMBDA], g["W"][O.THETA], g["W"][O.HV], cu, cv, u, dt, 30)
            assert rel_l2(srv.result(rid), ref) < 1e-5
    finally:
        srv.stop()


def test_wait_idle_means_every_request_is_done(ctx, grids):
    """The next batch is queued before the previous one completes; requests
    finishing with a batch still count until their results are delivered, so
    wait_idle returns only once every request is done and its result copied."""
    srv = R.Server(ctx)
    try:
        ids = []
        for k in range(14):
            g = grids[k % 2]
            p = R.heat_params(1.0, R.F32 if k % 3 else R.F64) if k % 2 else _bell_params(R.F32)
            u0 = _heat_u0(g, k) if k % 2 else _bell_u0(g, k)
            ids.append(srv.submit(g["grid"], p, u0, 1e-5 if k % 2 else BELL["dt"] / 20, 3 + 7 * k))
        srv.wait_idle(120)
        for rid in ids:
            done, status, _, _ = srv.poll(rid)
            assert done and status == 0, rid
            assert np.all(np.isfinite(srv.result(rid)))
        st = srv.stats()
        assert st["active"] == 0 and st["pending"] == 0 and st["completed"] == len(ids)
    finally:
        srv.stop()


def _need_fp32_heat(N):
    """Device bytes of a new FP32 heat bank (u, xa, xb, acc and the compensation
    of u, 8 columns each) and one I/O buffer."""
    return N * (5 * 8 * 4 + 8)


def test_request_that_can_never_fit_is_refused(ctx, grids):
    g = grids[1]
    held, _, total = ctx.mem_info()
    srv = R.Server(ctx, hbm_fraction=(held + _need_fp32_heat(g["N"]) // 2) / total)
    try:
        with pytest.raises(R.RbffdError) as e:
            srv.submit(g["grid"], R.heat_params(1.0, R.F32), _heat_u0(g, 0), 1e-5, 5)
        assert e.value.status == R.ERR_BUDGET
    finally:
        srv.stop()


def test_budget_for_one_request_serialises_admission(ctx, grids):
    g = grids[1]
    held, _, total = ctx.mem_info()
    # room for the server's bank table (64 KiB), one bank and one request's I/O
    # buffer (8 N bytes), not two: the next request waits for the first to leave
    srv = R.Server(ctx, hbm_fraction=(held + 65536 + _need_fp32_heat(g["N"]) + 4 * g["N"]) / total)
    try:
        u0 = [_heat_u0(g, k) for k in range(3)]
        ids = [srv.submit(g["grid"], R.heat_params(1.0, R.F32), u, 1e-5, 20) for u in u0]
        srv.wait_idle(60)
        outs = [srv.result(i) for i in ids]
        st = srv.stats()
        assert st["max_active_seen"] == 1 and st["completed"] == 3
        assert st["held_bytes"] <= st["budget_bytes"]
    finally:
        srv.stop()
    pde = R.HeatSphere(g["grid"], g["der"], 1.0, dtype=R.F32)
    pde.setShape(1, 128)
    for u, out in zip(u0, outs):
        pde.fillInitialConditions(u)
        pde.advance(R.RK4, 1e-5, 20)
        assert rel_l2(out, pde.getLocalSolution()) < 2e-6
    pde.close()


def test_shortest_first_admission(ctx, grids):
    """One slot, least work first: the request admitted at once runs first,
    then the waiting ones in order of work (grid nodes x stencil size x
    steps), whatever their arrival order; each result is the one it gets in
    arrival order."""
    g = grids[0]
    steps = [30, 40, 10, 20]
    u0 = [_heat_u0(g, k) for k in range(len(steps))]
    outs = {}
    for admission in ("arrival", "shortest"):
        srv = R.Server(ctx, max_active=1, admission=admission)
        try:
            srv.pause(True)
            ids, t_sub = [], []
            for u, k in zip(u0, steps):
                t_sub.append(time.perf_counter())
                ids.append(srv.submit(g["grid"], R.heat_params(1.0, R.F32), u, 1e-5, k))
            srv.pause(False)
            srv.wait_idle(60)
            done_at = []
            for rid, t in zip(ids, t_sub):
                done, status, lat, _ = srv.poll(rid)
                assert done and status == 0
                done_at.append(t + lat)
            outs[admission] = [srv.result(rid) for rid in ids]
        finally:
            srv.stop()
        order = [int(k) for k in np.argsort(done_at)]
        if admission == "shortest":
            # the first request takes the free slot as it arrives (unless the admission thread
            # first sees all four), then the waiting ones by work: 10, 20, 40 steps
            assert order in ([0, 2, 3, 1], [2, 3, 0, 1])
        else:
            assert order == [0, 1, 2, 3]
    for a, b in zip(outs["arrival"], outs["shortest"]):
        assert np.array_equal(a, b)
    with pytest.raises(ValueError):
        R.Server(ctx, admission="longest")


def test_cancel_pending_and_active(ctx, grids):
    g = grids[0]
    srv = R.Server(ctx, max_active=1)
    try:
        p = R.heat_params(1.0, R.F32)
        a = srv.submit(g["grid"], p, _heat_u0(g, 0), 1e-7, 2_000_000)  # runs until cancelled
        b = srv.submit(g["grid"], p, _heat_u0(g, 1), 1e-7, 10)         # waits for the slot
        t0 = time.time()
        while srv.poll(a)[3] < 0 and time.time() - t0 < 10:
            time.sleep(0.001)
        srv.cancel(b)
        assert srv.poll(b)[:2] == (True, R.ERR_CANCELLED)
        srv.cancel(a)
        assert srv.poll(a)[:2] == (True, R.ERR_CANCELLED)
        c = srv.submit(g["grid"], p, _heat_u0(g, 2), 1e-7, 10)
        assert srv.wait(c) == 0
        st = srv.stats()
        assert st["cancelled"] == 2 and st["completed"] == 1 and st["slots_reused"] >= 1
    finally:
        srv.stop()


def test_injected_admission_failure(ctx, grids):
    g = grids[0]
    srv = R.Server(ctx)
    try:
        srv.inject_admission_failures(1)
        p = R.heat_params(1.0, R.F32)
        a = srv.submit(g["grid"], p, _heat_u0(g, 0), 1e-5, 5)
        assert srv.wait(a) == R.ERR_OOM
        b = srv.submit(g["grid"], p, _heat_u0(g, 0), 1e-5, 5)
        assert srv.wait(b) == 0
        st = srv.stats()
        assert st["failed"] == 1 and st["completed"] == 1
    finally:
        srv.stop()


def test_malformed_and_trivial_requests(ctx, grids):
    g = grids[0]
    srv = R.Server(ctx)
    bare = R.Grid(ctx, g["xyz"], g["st"])  # no weights
    try:
        p = R.heat_params(1.0, R.F32)
        p.ntracers = 2
        with pytest.raises(R.RbffdError) as e:
            srv.submit(g["grid"], p, _heat_u0(g, 0), 1e-5, 5)
        assert e.value.status == -5
        with pytest.raises(R.RbffdError) as e:
            srv.submit(bare, R.heat_params(1.0, R.F32), _heat_u0(g, 0), 1e-5, 5)
        assert e.value.status == -6
        with pytest.raises(R.RbffdError) as e:
            srv.submit(g["grid"], R.heat_params(1.0, R.F32), _heat_u0(g, 0), 1e-5, -1)
        assert e.value.status == -1
        u0 = _heat_u0(g, 4)
        z = srv.submit(g["grid"], R.heat_params(1.0, R.F64), u0, 1e-5, 0)
        assert srv.wait(z) == 0 and np.array_equal(srv.result(z), u0)
    finally:
        srv.stop()
        bare.close()
