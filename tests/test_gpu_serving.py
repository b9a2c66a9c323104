"""Serving loop: continuous batching of independent LJ systems.

* a system's result is the same alone and in a mix (fixed tile width: bit-exact;
  autotuned widths: energies within 1e-10 relative, positions within 1e-6);
* the batched path agrees with the single-system mixed-precision driver and,
  within the precision form's bounds, with the FP64 oracle;
* admission respects the HBM budget (requests wait in FIFO order).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pd():
    from openfpm_pdata_b200 import pd as _pd
    _pd.lib()
    return _pd


def _sys(n, seed):
    from openfpm_pdata_b200 import workloads
    return workloads.serving_system(n, density=0.8, seed=seed)


def _serve(pd, systems, steps=20, autotune=False, tx=5, budget=8 << 30, slots=16, shapes=None):
    srv = pd.Server(budget, max_slots=slots, dt=0.005, skin=0.3, autotune=autotune, tx=tx)
    for bucket, shape in (shapes or {}).items():
        srv.set_shape(bucket, *shape)
    tickets = [srv.submit(x, v, L, steps) for (x, v, L) in systems]
    srv.run_until_done(tickets)
    out = [srv.result(t) for t in tickets]
    assert all(srv.state(t) == srv.DONE for t in tickets)
    _serve.last = srv
    return out, srv


def test_alone_equals_in_mix_bit_exact(pd):
    a = _sys(3000, 1)
    others = [_sys(n, 10 + k) for k, n in enumerate([700, 9000, 1500, 20000, 600])]
    (xa, Ea, _), = _serve(pd, [a])[0]
    mix, _ = _serve(pd, others[:2] + [a] + others[2:])
    xm, Em, _ = mix[2]
    assert np.array_equal(Ea, Em)
    assert np.array_equal(xa, xm)


def test_alone_vs_mix_autotuned(pd):
    a = _sys(4000, 2)
    others = [_sys(n, 20 + k) for k, n in enumerate([3500, 12000, 800])]
    (xa, Ea, _), = _serve(pd, [a], autotune=True)[0][:1]
    s1 = _serve.last
    mix, srv = _serve(pd, others + [a], autotune=True)
    xm, Em, _ = mix[-1]
    bucket = int(np.floor(np.log2(4000)))
    if s1.tuned()[bucket] == srv.tuned()[bucket]:
        assert np.array_equal(Ea, Em) and np.array_equal(xa, xm)
    else:
        # another tile width changes the FP32 summation order only
        np.testing.assert_allclose(Em[:, :3], Ea[:, :3], rtol=1e-6)
        d = xm - xa
        L = a[2]
        assert np.max(np.abs(d - np.round(d / L) * L)) < 1e-4
    assert len(srv.tuned()) >= 2


def test_served_matches_single_driver_and_oracle(pd, orc):
    x, v, L = _sys(6000, 3)
    (xs, Es, _), = _serve(pd, [(x, v, L)], steps=25, tx=5)[0]
    vd = pd.VectorDist(x.shape[0], np.zeros(3), np.full(3, L), np.ones(3, np.int32), 2.8, dtype=np.float64,
                       props=[(pd.PD_F32, 3), (pd.PD_F32, 3)])
    vd.hostToDevicePos(x)
    vd.hostToDeviceProp(0, v)
    md = pd.MD(vd, 0, 1, dt=0.005, skin=0.3, precision=pd.PREC_MIXED)
    md.set_tiles(True, tx=5, threads_per_particle=2)
    E1 = md.run(25)
    # same tile width and lanes: the same trajectory; sums of the energies differ in order only
    np.testing.assert_allclose(Es[:, :3], E1[:, :3], rtol=1e-12, atol=1e-12)
    assert np.array_equal(Es[:, 3], E1[:, 3])
    x1 = np.zeros_like(x)
    x1[vd.gid(with_ghost=False)] = vd.deviceToHostPos(with_ghost=False)
    assert np.array_equal(x1, xs)
    _, _, Eo = orc.md_lj(x, v, np.zeros(3), np.full(3, L), np.ones(3, np.int32), 2.8, 2.5, 0.3, 1.0, 1.0, 0.005,
                         1.0, 25)
    tot = Es[:, 0] + Es[:, 1]
    toto = Eo[1:, 0] + Eo[1:, 1]
    assert np.max(np.abs(tot - toto) / np.abs(toto)) < 2e-5


@pytest.mark.parametrize("lanes,block", [(1, 128), (4, 256), (2, 128)])
def test_served_shape_matches_single_driver(pd, lanes, block):
    """Every launch shape of the batched force kernel (lanes per particle, CTA size)
    gives the single-system driver's trajectory with the same shape, bit for bit."""
    x, v, L = _sys(6000, 3)
    bucket = int(np.floor(np.log2(6000)))
    (xs, Es, _), = _serve(pd, [(x, v, L)], steps=15, autotune=True, shapes={bucket: (5, lanes, block)})[0]
    assert _serve.last.tuned()[bucket] == (5, lanes, block)
    vd = pd.VectorDist(x.shape[0], np.zeros(3), np.full(3, L), np.ones(3, np.int32), 2.8, dtype=np.float64,
                       props=[(pd.PD_F32, 3), (pd.PD_F32, 3)])
    vd.hostToDevicePos(x)
    vd.hostToDeviceProp(0, v)
    md = pd.MD(vd, 0, 1, dt=0.005, skin=0.3, precision=pd.PREC_MIXED)
    md.set_tiles(True, tx=5, threads_per_particle=lanes)
    md.set_block(block)
    E1 = md.run(15)
    np.testing.assert_allclose(Es[:, :3], E1[:, :3], rtol=1e-12, atol=1e-12)
    x1 = np.zeros_like(x)
    x1[vd.gid(with_ghost=False)] = vd.deviceToHostPos(with_ghost=False)
    assert np.array_equal(x1, xs)


def test_mixed_shapes_alone_equals_in_mix(pd):
    """Systems of different size buckets with different shapes (both CTA sizes, all
    lane counts) in one batch: each result equals the system served alone."""
    systems = [_sys(n, 50 + k) for k, n in enumerate([700, 3000, 9000, 20000])]
    shapes = {9: (5, 1, 128), 11: (7, 4, 256), 13: (9, 2, 128), 14: (5, 2, 256)}
    mix, _ = _serve(pd, systems, shapes=shapes)
    for k, s in enumerate(systems):
        (xa, Ea, _), = _serve(pd, [s], shapes=shapes)[0]
        assert np.array_equal(Ea, mix[k][1]) and np.array_equal(xa, mix[k][0])


def test_admission_by_budget(pd):
    systems = [_sys(n, 30 + k) for k, n in enumerate([20000, 20000, 20000])]
    # a budget for about one system at a time: the others wait, all finish
    srv = pd.Server(int(20000 * 700 * 1.5) + (8 << 20), max_slots=8, dt=0.005, skin=0.3, autotune=False, tx=5)
    tickets = [srv.submit(x, v, L, 10) for (x, v, L) in systems]
    active, queued = srv.tick()
    assert active == 1 and queued == 2
    srv.run_until_done(tickets)
    times = [srv.result(t)[2] for t in tickets]
    assert times[0][2] <= times[1][1] and times[1][2] <= times[2][1]   # FIFO, one at a time
    assert srv.stats()["systems_done"] == 3


def test_staging_paths_alone_equals_in_mix(pd):
    # a 512 MB budget: 8 MB upload ring and download buffer, 16 MB inbox and
    # outbox.  Six finished systems that are not released hold 14.4 MB of the
    # outbox; then the 350k system uploads through staging of its own (it does not
    # fit the inbox) and retires through the grown download buffer, the 120k
    # system through the download buffer, the 60k system through the outbox.
    # Every result equals the system served alone, bit for bit.
    fillers = [_sys(100000, 70 + k) for k in range(6)]
    systems = [_sys(n, 40 + k) for k, n in enumerate([350000, 120000, 60000])]
    srv = pd.Server(512 << 20, max_slots=4, dt=0.005, skin=0.3, autotune=False, tx=5)
    held = [srv.submit(x, v, L, 10) for (x, v, L) in fillers]
    srv.run_until_done(held)
    tickets = [srv.submit(x, v, L, 10) for (x, v, L) in systems]
    srv.run_until_done(tickets)
    for t, s in zip(tickets + held, systems + fillers):
        xm, Em, _ = srv.result(t)
        (xa, Ea, _), = _serve(pd, [s], steps=10, budget=512 << 20, slots=4)[0]
        assert np.array_equal(Em, Ea)
        assert np.array_equal(xm, xa)
        assert xm.shape == s[0].shape and np.all(np.isfinite(xm))


def test_inbox_wraps_and_falls_back(pd):
    # 16 MB inbox: the first wave fills it (the last systems fall back to host
    # copies), the second wave is submitted while the first runs and reuses the
    # regions freed by its admissions; every result equals the system served alone
    rng = np.random.default_rng(5)
    sizes = [int(n) for n in rng.integers(20000, 60000, size=18)]
    systems = [_sys(n, 60 + k) for k, n in enumerate(sizes)]
    srv = pd.Server(512 << 20, max_slots=4, dt=0.005, skin=0.3, autotune=False, tx=5)
    tickets = [srv.submit(x, v, L, 10) for (x, v, L) in systems[:12]]
    for _ in range(6):
        srv.tick()
    tickets += [srv.submit(x, v, L, 10) for (x, v, L) in systems[12:]]
    srv.run_until_done(tickets)
    for t, s in zip(tickets, systems):
        xm, Em, _ = srv.result(t)
        (xa, Ea, _), = _serve(pd, [s], steps=10, budget=512 << 20, slots=4)[0]
        assert np.array_equal(Em, Ea)
        assert np.array_equal(xm, xa)
    # results released out of order free the outbox from its oldest region on;
    # a third wave then retires into the freed space
    for t in reversed(tickets):
        srv.release(t)
    third = systems[:6]
    t3 = [srv.submit(x, v, L, 10) for (x, v, L) in third]
    srv.run_until_done(t3)
    for t, s in zip(t3, third):
        xm, Em, _ = srv.result(t)
        (xa, Ea, _), = _serve(pd, [s], steps=10, budget=512 << 20, slots=4)[0]
        assert np.array_equal(Em, Ea)
        assert np.array_equal(xm, xa)


def test_result_and_release_follow_the_request_state(pd):
    # a result is refused until the system is done (PD_ESTATE), a release until it
    # is done or failed; after the release the ticket is unknown; the result read
    # twice from the outbox is the same
    srv = pd.Server(1 << 30, max_slots=2, dt=0.005, skin=0.3, autotune=False, tx=5)
    x, v, L = _sys(3000, 90)
    t = srv.submit(x, v, L, 5)
    with pytest.raises(pd.PdError):
        srv.result(t)
    with pytest.raises(pd.PdError):
        srv.release(t)
    srv.run_until_done([t])
    x1, E1, _ = srv.result(t)
    x2, E2, _ = srv.result(t)
    assert np.array_equal(x1, x2) and np.array_equal(E1, E2)
    srv.release(t)
    with pytest.raises(pd.PdError):
        srv.release(t)
