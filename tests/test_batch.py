"""The batched and served forms (ablsteadyrans_b200.batch, .serve): many
independent instances on one GPU, each with its own stream, context and
resident state. A result is the same alone and in the mix, bit for bit; the
server admits by device footprint and finishes every request."""
import numpy as np
import pytest

from ablsteadyrans_b200 import batch, serve, workloads


def test_config3_instances_follow_the_configuration():
    insts = batch.config3(count=6, seed=3)
    assert len(insts) == 6
    for inst in insts:
        g = inst.grid
        assert g.nx == g.ny and g.nx in batch.CONFIG3_SIZES and g.nz in batch.CONFIG3_LAYERS
        assert g.dx == 30.0 and not g.periodic_x and not g.periodic_y
        assert 0.2 <= inst.ustar <= 0.6 and 0.01 <= inst.z0 <= 0.5
    # seeded: the same draw twice
    again = batch.config3(count=6, seed=3)
    assert [i.name for i in insts] == [i.name for i in again]
    assert all(np.array_equal(a.z, b.z) for a, b in zip(insts, again))


def test_config4_requests_are_an_open_loop_poisson_process():
    reqs = serve.requests_config4(200, rate=5.0, seed=1, sizes=(32,), layers=(16,))
    t = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(t) > 0)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert 0.15 < gaps.mean() < 0.25          # 1 / rate
    frac = np.mean([r.kind == "init" for r in reqs])
    assert 0.6 < frac < 0.8                   # 70 % mass-consistent only


def _small(seed, n, nz, precision):
    return workloads.tile(n, nz, seed, precision=precision)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_gpu_member_same_alone_and_in_the_mix(precision):
    """Three members iterated one by one and then, from the same start,
    together on concurrent threads and streams: identical fields, bit for bit."""
    shapes = [(32, 24), (48, 32), (40, 24)]
    alone = batch.Batch([_small(s, n, nz, precision) for s, (n, nz) in enumerate(shapes)])
    alone.run(3, concurrent=False)
    ref = [m.fields() for m in alone.members]
    alone.close()
    mix = batch.Batch([_small(s, n, nz, precision) for s, (n, nz) in enumerate(shapes)])
    mix.run(3, concurrent=True)
    got = [m.fields() for m in mix.members]
    mix.close()
    for r, g_ in zip(ref, got):
        for f in r:
            assert np.array_equal(r[f], g_[f]), f
        assert np.abs(r["u"]).max() > 0


@pytest.mark.gpu
def test_gpu_server_admits_by_footprint_and_finishes_every_request():
    """Requests arriving together under a budget of about two requests: all
    are served, never more than the budget resident at once, and each
    result equals the same request served alone."""
    peak, vol = serve.measure_peak_bytes(32, 16)
    model = (0.0, peak / vol)
    reqs = serve.requests_config4(6, rate=100.0, seed=2, sizes=(32,), layers=(16,))
    for r in reqs[:2]:
        r.kind = "rans"
    srv = serve.Server(budget=2.5 * peak, footprint=model, max_iterations=5)
    srv.run(reqs)
    assert all(r.done is not None and r.latency > 0 for r in reqs)
    assert all(r.status in ("initialized", "running", "steady") for r in reqs), [r.status for r in reqs]
    assert srv.peak_active <= 2
    # the same requests alone
    for r in reqs:
        alone = serve.requests_config4(6, rate=100.0, seed=2, sizes=(32,), layers=(16,))[r.id]
        alone.kind = r.kind
        srv1 = serve.Server(budget=1e15, footprint=model, max_iterations=5)
        srv1.run([alone])
        assert alone.status == r.status and alone.iterations == r.iterations
        if r.kind == "init":
            assert alone.result == r.result


@pytest.mark.gpu
def test_gpu_native_driver_equals_the_python_driver():
    """The C++ driver (gb_driver: local dtau, iteration, criterion, SER law)
    takes the same steps as the Python one: identical fields after 8 steps."""
    a = batch.Batch([_small(7, 32, 24, 0)])
    for _ in range(8):
        a.members[0].step()
    ref = a.members[0].fields()
    hist = [h[0] for h in a.members[0].driver.history]
    a.close()
    b = batch.Batch([_small(7, 32, 24, 0)])
    cfls = []
    for _ in range(8):
        verdict, info, cfl = b.members[0].native.step()
        cfls.append(cfl)
    got = b.members[0].fields()
    b.close()
    assert cfls == hist
    for f in ref:
        assert np.array_equal(ref[f], got[f]), f


@pytest.mark.gpu
def test_gpu_native_batch_same_alone_and_in_the_mix():
    shapes = [(32, 24), (48, 32), (40, 24)]
    one = batch.Batch([_small(s, n, nz, 1) for s, (n, nz) in enumerate(shapes)])
    one.run_native(4, threads=1)
    ref = [m.fields() for m in one.members]
    one.close()
    mix = batch.Batch([_small(s, n, nz, 1) for s, (n, nz) in enumerate(shapes)])
    mix.run_native(4, threads=0)
    got = [m.fields() for m in mix.members]
    assert all(m.iterations == 4 for m in mix.members)
    mix.close()
    for r, g_ in zip(ref, got):
        for f in r:
            assert np.array_equal(r[f], g_[f]), f


def test_sequential_latencies_are_a_fifo_queue():
    """The plain FP64 sequential path's latencies: one request at a time in
    arrival order, each starting when it has arrived and the previous one
    is done."""
    from ablsteadyrans_b200.serve import sequential_latencies
    assert sequential_latencies([0.0, 1.0, 1.5, 10.0], [2.0, 2.0, 2.0, 1.0]) == [2.0, 3.0, 4.5, 1.0]
    assert sequential_latencies([], []) == []


def test_config4_tiles_do_not_depend_on_the_arrival_rate():
    """The served sweep measures each request's sequential FP64 service time
    once and replays the FIFO queue at every rate: that holds because the
    same seed draws the same tiles and kinds at any rate (only the arrival
    times scale, by 1 / rate)."""
    a = serve.requests_config4(8, rate=0.5, seed=3, sizes=(32, 48), layers=(16, 24))
    b = serve.requests_config4(8, rate=20.0, seed=3, sizes=(32, 48), layers=(16, 24))
    for x, y in zip(a, b):
        assert x.kind == y.kind
        assert (x.inst.grid.nx, x.inst.grid.ny, x.inst.grid.nz) == (y.inst.grid.nx, y.inst.grid.ny, y.inst.grid.nz)
        assert np.array_equal(x.inst.z, y.inst.z)
        assert x.arrival * 0.5 == pytest.approx(y.arrival * 20.0, rel=1e-12)
